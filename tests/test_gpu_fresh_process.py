"""A fresh process whose first call captures a CUDA graph: the one-time
per-device set-up of the batch kernels (decode-plan tables, shared-memory
limits) synchronises, so it must run before the capture starts, not inside
it.  Earlier tests in one pytest process would hide this, hence the child
process."""
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

CHILD = r'''
import sys
import numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/tests")
import torch
import scrs_b200
from scrs_b200.api import Api, Library
from scrs_b200.batch import StripeBatch
from scenarios import device_stripes, make_mixed_batch
from conftest import build_oracle

oracle = Api(Library(build_oracle(), prefix="oracle_", device=False))
gpu = scrs_b200.api_default()
specs, rng = make_mixed_batch(torch, 64, 41, lens=(1024, 4096))
stripes, outs, expect, keep = device_stripes(torch, oracle, specs, rng)
torch.cuda.synchronize()
b = StripeBatch(gpu.lib, len(stripes))
b.set(stripes)
b.run(graph=True)  # the first device work of the process, inside a capture
torch.cuda.synchronize()
b.check()
bad = [i for i, (o, e) in enumerate(zip(outs, expect)) if not np.array_equal(o.cpu().numpy(), e)]
print("mismatched stripes:", bad)
sys.exit(1 if bad else 0)
'''


def test_first_call_of_a_process_is_a_graph_run():
    r = subprocess.run([sys.executable, "-c", CHILD, str(ROOT)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout[-3000:], r.stderr[-3000:])
