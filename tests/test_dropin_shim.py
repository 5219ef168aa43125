"""The C++ drop-in shim (include/dynasor_b200_dropin.hpp), compiled against
the reference's headers into oracle/_ref/dropin_verify: the reference's
--verify flow (spmttkrp_reference vs the GPU sweep through GpuSweep,
compare_factors_detail within 1e-4) and cpals_gpu against the reference's
cpals from the same seed.  On a machine without a GPU the same binary
stops with the library's no-device error (no CPU fallback)."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, HAS_GPU

EXE = os.path.join(ROOT, "oracle", "_ref", "dropin_verify")


def _write_tns(path, dims, vals, idx):
    with open(path, "w") as f:
        for i in range(len(vals)):
            f.write(f"{idx[0][i] + 1} {idx[1][i] + 1} {idx[2][i] + 1} {vals[i]:.9g}\n")


@pytest.fixture
def tns(tmp_path):
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/dropin_verify not built (needs the reference tree at build time)")
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.zipf((3000, 700, 200), draws=60000, s=1.1, seed=5)
    p = tmp_path / "zipf.tns"
    _write_tns(p, dims, vals, idx)
    return str(p)


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device error path")
def test_shim_fails_loudly_without_a_device(tns):
    r = subprocess.run([EXE, tns, "16", "4", "7", "3"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 2, r.stdout + r.stderr
    assert "no CUDA device" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("rank,threads", [(16, 4), (32, 8)])
def test_reference_verify_flow_through_the_shim(tns, rank, threads):
    r = subprocess.run([EXE, tns, str(rank), str(threads), "7", "6"], capture_output=True,
                       text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PASS: Frobenius relative error" in r.stdout
    assert "PASS: cpals_gpu" in r.stdout
