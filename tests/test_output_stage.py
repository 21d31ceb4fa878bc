"""The output stage (xb_image_to_rgb8, xb_write_png, xb_image_noise_stats): host code, no GPU.

Against golden vectors computed by the reference itself (tests/golden/output.npz from
gen_golden.py: its ImageNoiseEstimator and save_image's 8-bit values, for seeded images, edge
cases and its own converged config-1 render): the statistics bit for bit, the pixels exactly
(flipped as the reference flips them on write). The PNG is decoded here with zlib and checked
chunk by chunk."""
import os
import struct
import zlib

import numpy as np
import pytest

import xenon_b200 as xb

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "output.npz"))
NAMES = sorted({k.rsplit("_", 1)[0] for k in GOLD.files})
FIELDS = ("mean_squared_score", "rms_score", "mean_absolute", "median_absolute", "p95_absolute",
          "max_absolute", "avg_luminance", "edge_threshold", "epsilon", "valid_pixel_ratio")


@pytest.mark.parametrize("name", NAMES)
def test_noise_stats_match_the_reference(name):
    got = xb.noise_stats(GOLD[f"{name}_image"])
    want = GOLD[f"{name}_stats"]
    mine = np.array([got[k] for k in FIELDS], np.float32)
    assert np.array_equal(mine.view(np.uint32), want.view(np.uint32)), (name, mine, want)
    assert (got["valid_pixel_count"], got["total_interior_pixel_count"]) == tuple(GOLD[f"{name}_counts"])


@pytest.mark.parametrize("name", NAMES)
def test_8bit_pixels_match_the_reference(name):
    # the reference converts its framebuffer row by row and flips it on write
    assert np.array_equal(xb.image_to_rgb8(GOLD[f"{name}_image"]), GOLD[f"{name}_rgb8"][::-1])


def _chunks(data: bytes):
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, out = 8, []
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        kind, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        (crc,) = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert crc == zlib.crc32(kind + body), kind
        out.append((kind, body))
        pos += 12 + n
    return out


@pytest.mark.parametrize("shape", [(48, 64), (1, 1), (3, 30000)])   # 90,001-byte rows: two stored blocks
def test_png_decodes_to_the_8bit_pixels(tmp_path, shape):
    img = np.random.default_rng(3).random(shape + (3,)).astype(np.float32) * 1.2 - 0.1
    path = tmp_path / "out.png"
    xb.write_png(str(path), img)
    chunks = _chunks(path.read_bytes())
    assert [k for k, _ in chunks] == [b"IHDR", b"IDAT", b"IEND"]
    w, h, depth, ctype, comp, filt, inter = struct.unpack(">IIBBBBB", chunks[0][1])
    assert (w, h, depth, ctype, comp, filt, inter) == (shape[1], shape[0], 8, 2, 0, 0, 0)
    raw = zlib.decompress(chunks[1][1])
    rows = np.frombuffer(raw, np.uint8).reshape(h, 1 + 3 * w)
    assert np.all(rows[:, 0] == 0)
    assert np.array_equal(rows[:, 1:].reshape(h, w, 3), xb.image_to_rgb8(img))


def test_bad_arguments_and_paths_fail_loudly(tmp_path):
    img = np.zeros((4, 4, 3), np.float32)
    with pytest.raises(xb.XenonError):
        xb.write_png(str(tmp_path / "missing_dir" / "x.png"), img)
    with pytest.raises(xb.XenonError):
        xb.noise_stats(np.zeros((0, 4, 3), np.float32))


def test_cpp_face_save_image(tmp_path):
    """csrc/b200_renderer.h compiles as C++17 against the library, and its save_image writes the
    same file and statistics as the C entry points (host code only: no renderer is created)."""
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    img = GOLD["noisy_gradient_image"]
    h, w = img.shape[:2]
    (tmp_path / "img.bin").write_bytes(np.ascontiguousarray(img, np.float32).tobytes())
    (tmp_path / "t.cpp").write_text(f"""
#include <cstdio>
#include <fstream>
#include <vector>
#include "b200_renderer.h"
int main() {{
  std::vector<float> img({w} * {h} * 3);
  std::ifstream("img.bin", std::ios::binary).read(reinterpret_cast<char*>(img.data()), img.size() * 4);
  const xb_noise_stats s = xb::B200Renderer::save_image("cpp.png", img.data(), {w}, {h});
  std::printf("%a %d\\n", s.mean_squared_score, s.valid_pixel_count);
  try {{
    xb::B200Renderer::save_image("no_such_dir/x.png", img.data(), {w}, {h});
  }} catch (const xb::Error& e) {{
    std::printf("error %d\\n", e.code);
  }}
  return 0;
}}
""")
    lib = os.path.join(root, "xenon_b200", "lib")
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(root, "xenon_b200", "csrc"), "t.cpp", "-o", "t",
                    "-L", lib, "-lxenon_b200", f"-Wl,-rpath,{lib}"], cwd=tmp_path, check=True)
    out = subprocess.run(["./t"], cwd=tmp_path, check=True, capture_output=True, text=True).stdout.split()
    stats = xb.noise_stats(img)
    assert float.fromhex(out[0]) == float(np.float32(stats["mean_squared_score"])) and int(out[1]) == stats["valid_pixel_count"]
    assert out[2:] == ["error", str(-5)]                    # XB_E_IO
    xb.write_png(str(tmp_path / "py.png"), img)
    assert (tmp_path / "cpp.png").read_bytes() == (tmp_path / "py.png").read_bytes()


def test_png_from_8bit_pixels_equals_png_from_the_image(tmp_path):
    """xb_write_png_rgb8 over xb_image_to_rgb8's pixels writes the same file as xb_write_png."""
    import xenon_b200 as xb
    rng = np.random.default_rng(4)
    img = (rng.random((37, 53, 3)) * 1.3 - 0.1).astype(np.float32)
    a, b = tmp_path / "a.png", tmp_path / "b.png"
    xb.write_png(str(a), img)
    xb.write_png_rgb8(str(b), xb.image_to_rgb8(img))
    assert a.read_bytes() == b.read_bytes()
