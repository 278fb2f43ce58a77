"""Model files (io::ply, src/io/ply.rs:35-303) through the C ABI: the device
packs / unpacks the records, and the files must match the oracle's byte for
byte (save) or decode to the same records bit for bit (load)."""
import struct

import numpy as np
import pytest

import oracle as O
import rgsplat_b200 as R
from rgsplat_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return R.Context()


def model(n=1000, seed=41):
    g = scenes.random_gaussians(n, seed, 1.5, (-3.5, 0.7), (0.0, 1.5))
    g[::7, 4:8] *= 3.0        # unnormalised rotations
    g[5, 4:8] = 0.0           # degenerate quaternion -> identity in .splat
    g[6, 3] = 40.0            # saturated opacity byte
    g[7, 11] = -10.0          # clamped colour byte
    return g


def test_save_ply_matches_reference_bytes(ctx, tmp_path):
    g = model()
    p = tmp_path / "sub" / "model.ply"  # the parent is created, as the reference does
    R.save_ply(g, p, ctx=ctx)
    assert p.read_bytes() == O.save_ply_bytes(g)


def test_save_splat_matches_reference_bytes(ctx, tmp_path):
    g = model()
    p = tmp_path / "model.splat"
    R.save_splat(g, p, ctx=ctx)
    data = p.read_bytes()
    assert len(data) == 32 * g.shape[0]
    assert data == O.save_splat_bytes(g)


def test_load_ply_binary_roundtrip_and_variants(ctx, tmp_path):
    g = model(777)
    p = tmp_path / "m.ply"
    p.write_bytes(O.save_ply_bytes(g))
    back = R.load_ply(p, ctx=ctx)
    assert np.array_equal(back.view(np.uint32), g.view(np.uint32))
    # big-endian, mixed widths, shuffled order, unknown property, partial SH
    rng = np.random.default_rng(3)
    props = [("double", "z"), ("float", "x"), ("uchar", "opacity"), ("ushort", "scale_2"), ("float", "rot_1"),
             ("int", "f_rest_30"), ("float", "nx"), ("float", "f_dc_2"), ("float", "y")]
    fmt = {"float": "f", "double": "d", "uchar": "B", "ushort": "H", "int": "i"}
    n = 300
    for order in (">", "<"):
        head = (f"ply\nformat {'binary_big_endian' if order == '>' else 'binary_little_endian'} 1.0\n"
                f"element vertex {n}\n" + "".join(f"property {t} {nm}\n" for t, nm in props) + "end_header\n").encode()
        body = b""
        for _ in range(n):
            for t, _nm in props:
                v = int(rng.integers(0, 255)) if t in ("uchar", "ushort", "int") else float(rng.normal())
                body += struct.pack(order + fmt[t], v)
        data = head + body
        p.write_bytes(data)
        got = R.load_ply(p, ctx=ctx)
        want = O.load_ply_bytes(data)
        assert got.shape == (n, 59)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_load_ply_ascii(ctx, tmp_path):
    lines = ["ply", "format ascii 1.0", "element vertex 3", "property float x", "property float opacity",
             "property float f_rest_1", "end_header", "1.5 -0.25 0.125", "2 bad 3", ""]
    data = "\n".join(lines).encode()
    p = tmp_path / "a.ply"
    p.write_bytes(data)
    got = R.load_ply(p, ctx=ctx)
    assert np.array_equal(got.view(np.uint32), O.load_ply_bytes(data).view(np.uint32))
    assert got.shape[0] == 3 and got[1, 3] == 0.0 and got[2, 0] == 0.0  # unparsable -> 0, missing line -> defaults


def test_load_ply_errors(ctx, tmp_path):
    p = tmp_path / "x.ply"
    p.write_bytes(b"not a ply\n")
    with pytest.raises(R.RgsError):
        R.load_ply(p, ctx=ctx)
    p.write_bytes(b"ply\nformat binary_little_endian 1.0\nelement vertex 5\nproperty float x\nend_header\n" + b"\0" * 8)
    with pytest.raises(R.RgsError):  # body shorter than its vertex count
        R.load_ply(p, ctx=ctx)
    with pytest.raises(R.RgsError):
        R.load_ply(tmp_path / "missing.ply", ctx=ctx)


def test_trainer_save_and_load(tmp_path):
    g = model(2000)
    cams = scenes.sphere_cameras(2, 4.0, [(64, 48)], 1.2)
    tr = R.Trainer(g, cams)
    tr.save_ply(tmp_path / "t.ply")
    assert (tmp_path / "t.ply").read_bytes() == O.save_ply_bytes(g)
    tr.save_splat(tmp_path / "t.splat")
    assert (tmp_path / "t.splat").read_bytes() == O.save_splat_bytes(g)
    h = model(1500, seed=42)
    (tmp_path / "h.ply").write_bytes(O.save_ply_bytes(h))
    assert tr.load_ply(tmp_path / "h.ply") == 1500
    assert np.array_equal(tr.gaussians().view(np.uint32), h.view(np.uint32))
    assert tr.adam_state().t == 0
