"""The viewer's data preparation and the oracle of its deferred shading, on CPU.

  * pack_face_color_lut / quantize_lut / extract_mlp_weights of the package
    against fixtures made by the reference's own functions
    (tests/golden/make_golden_viewer.py), bit for bit;
  * the oracle's restatement of the viewer's shader arithmetic against the
    pinned oracle: its LUT interpolation equals the multires interpolation of
    the same texels (multires.cu:224-247, the lattice the shader restates) and
    its view-direction SH2 equals encode_view_dir_sh2 (encoding.cu:89-130);
  * the renderer refuses to run anywhere but on the GPU.
"""

import os

import numpy as np
import pytest
import torch

from diffsoup_b200 import viewer
from oracle import cpu
from oracle import viewer as oviewer

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "viewer_lut.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("case", ["small", "rows", "clip"])
def test_lut_packing_matches_reference(golden, case):
    feat, alpha, level = golden[f"{case}_feat"], golden[f"{case}_alpha"], int(golden[f"{case}_level"])
    lut = viewer.pack_face_color_lut(feat, alpha, feat.shape[0], level)
    assert lut.dtype == torch.float32
    assert np.array_equal(lut.numpy(), golden[f"{case}_lut"])
    lut0, lut1 = viewer.quantize_lut(lut)
    assert np.array_equal(lut0.numpy(), golden[f"{case}_lut0"])
    assert np.array_equal(lut1.numpy(), golden[f"{case}_lut1"])
    assert viewer.level_size(level) == oviewer.level_size(level) == feat.shape[1]


def test_mlp_extraction_matches_reference(golden):
    sd = {k[3:]: torch.from_numpy(golden[k]) for k in golden.files if k.startswith("sd_")}
    sd = dict(sorted(sd.items(), key=lambda kv: (int(kv[0].split(".")[1]), kv[0].endswith("bias"))))
    got = viewer.extract_mlp_weights(sd)
    for name, g in zip(("W1", "b1", "W2", "b2", "W3", "b3"), got):
        assert np.array_equal(g.numpy(), golden[f"mlp_{name}"]), name
    packed = viewer.pack_mlp(*got)
    assert packed.numel() == viewer.MLP_PARAMS == 595


def _gbuf(rng, B, H, W, T, empty=0.3):
    """Random G-buffer: barycentrics in the triangle, ids in [1, T], some empty."""
    b = rng.dirichlet([1.0, 1.0, 1.0], size=(B, H, W)).astype(np.float32)
    g = np.zeros((B, H, W, 4), np.float32)
    g[..., 0], g[..., 1] = b[..., 0], b[..., 1]
    g[..., 2] = rng.uniform(-1, 1, (B, H, W))
    ids = rng.integers(1, T + 1, (B, H, W))
    ids[rng.random((B, H, W)) < empty] = 0
    g[..., 3] = ids.astype(np.float32)
    return g


@pytest.mark.parametrize("level", [0, 2, 5])
def test_oracle_lut_interpolation_is_the_multires_lattice(level):
    rng = np.random.default_rng(level)
    T, S = 9, oviewer.level_size(level)
    lut0 = rng.integers(0, 256, (T * S + 5, 4), dtype=np.uint8)
    lut1 = rng.integers(0, 256, (T * S + 5, 4), dtype=np.uint8)
    g = _gbuf(rng, 2, 12, 10, T)
    A, Bv, mask = oviewer.geometry_pass(g, level, lut0, lut1)
    feat = np.concatenate([lut0[:T * S], lut1[:T * S]], -1).astype(np.float64).reshape(T, S, 8) / 255.0
    want = cpu.multires_color(g, level, level, feat, precision="f64")
    assert np.array_equal(mask, g[..., 3] > 0)
    np.testing.assert_allclose(A[mask], want[..., :4][mask], rtol=0, atol=1e-12)
    np.testing.assert_allclose(Bv[mask], want[..., 4:7][mask], rtol=0, atol=1e-12)


def test_oracle_view_encoding_is_encode_view_dir_sh2():
    rng = np.random.default_rng(3)
    from diffsoup_b200 import scenes
    sc = scenes.make_scene(1, seed=2, num_tris=10, resolution=(24, 20), with_targets=False)
    inv = sc.inv_mvps()
    g = _gbuf(rng, inv.shape[0], 24, 20, 10, empty=0.0)
    got = oviewer.sh2(oviewer.view_dirs(inv.shape[0], 24, 20, inv))
    want = cpu.encode_view(g, inv, sh=True, precision="f64")
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-9)


def test_oracle_rgba8_rounding():
    c = np.array([[0.0, 1.0, 0.5], [-0.2, 1.7, 0.501], [np.float32(0.5 / 255), np.float32(1.5 / 255), 0.998]],
                 np.float32)
    q = oviewer.to_rgba8(c)
    assert q[..., 3].tolist() == [255, 255, 255]
    assert q[0, :3].tolist() == [0, 255, 128] and q[1, :3].tolist() == [0, 255, 128]


def test_renderer_is_gpu_only(golden):
    lut0, lut1 = golden["small_lut0"], golden["small_lut1"]
    verts = np.zeros((3, 3), np.float32)
    faces = np.array([[0, 1, 2]], np.int32)
    W = [np.zeros((16, 16), np.float32), np.zeros(16, np.float32)] * 2 + [np.zeros((3, 16), np.float32),
                                                                          np.zeros(3, np.float32)]
    with pytest.raises(RuntimeError, match="GPU only"):
        viewer.Renderer(verts, faces, lut0, lut1, *W, level=2, device="cpu")
    with pytest.raises(RuntimeError, match="headless"):
        viewer.launch_viewer()


def test_png_writer_round_trip(tmp_path):
    """viewer._write_png (the screenshots of benchmark()) as a standard PNG:
    signature, IHDR, CRCs, and the pixel rows back through zlib."""
    import struct
    import zlib

    rng = np.random.default_rng(0)
    img = rng.integers(0, 256, (5, 7, 4), dtype=np.uint8)
    path = tmp_path / "x.png"
    viewer._write_png(str(path), img)
    data = path.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, chunks = 8, {}
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        tag, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        crc = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]
        assert crc == zlib.crc32(tag + body) & 0xFFFFFFFF
        chunks[tag] = body
        pos += 12 + n
    w, h, depth, ctype = struct.unpack(">IIBB", chunks[b"IHDR"][:10])
    assert (w, h, depth, ctype) == (7, 5, 8, 6)
    raw = zlib.decompress(chunks[b"IDAT"])
    rows = np.frombuffer(raw, np.uint8).reshape(5, 1 + 7 * 4)
    assert (rows[:, 0] == 0).all()
    assert np.array_equal(rows[:, 1:].reshape(5, 7, 4), img)
    assert b"IEND" in chunks
