"""The persistent bulk-copy (TMA) plane kernels (opt-in with CFFT_TMA=fwd|all) and their
bounded waits.  The switch is read once per process, so the cases (tests/tma_cases.py)
run in a child process with CFFT_TMA=all: headline-batch parity of both bulk-copy plane
stages against FP64 truth, the forward kernel with interaction factors in the Ia-3d
96^3 diffusion step against the FP64 oracle, and the bounded-wait timeout path."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)


def test_bulk_copy_plane_kernels():
    here = os.path.dirname(os.path.abspath(__file__))
    env = dict(os.environ, CFFT_TMA="all")
    r = subprocess.run([sys.executable, os.path.join(here, "tma_cases.py")], env=env, capture_output=True, text=True,
                       timeout=900)
    print(r.stdout[-3000:])
    assert r.returncode == 0 and "TMA_CASES_OK" in r.stdout, r.stderr[-3000:]
