"""The table-driven Hilbert index (two levels per lookup) against the bitwise encoder, and the table-driven node
corner decoder against the bitwise decoder, on the host (no GPU).

The cubic-box key kernels use the encoding table, and the node geometry of cubic boxes (MAC radii, group boxes) the
decoding table; the GPU parity tests compare keys and MAC radii with the oracle. This check compiles the shared
header for the host and compares the encoders on edge cases, 2M random cells and every combination of the six
lowest bits, and the decoders at every level on edge cases and 200k random cells.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    return None


def test_hilbert_table_equals_bitwise_encoder(tmp_path):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not available")
    exe = str(tmp_path / "hilbert_table_check")
    subprocess.run([nvcc, "-std=c++17", "-O2", "--expt-relaxed-constexpr",
                    "-I" + os.path.join(ROOT, "ryoanji_b200", "csrc"), "-I" + os.path.join(ROOT, "include"),
                    os.path.join(HERE, "hilbert_table_check.cu"), "-o", exe], check=True, capture_output=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 mismatches" in r.stdout
