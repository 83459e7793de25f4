"""The drop-in proven from the reference's side: the reference library built
with the CUDA branch of integration/vp9_decoder_cuda.patch decodes packets
through its own public API — cvp9_create(CVP9_BACKEND_CUDA), cvp9_decode,
cvp9_get_frame / cvp9_get_frame_sync — and every frame equals the same
library's CPU backend (the reference's own reconstruction), byte for byte,
with the CVP9_ERR_AGAIN back-pressure loop of the reference's VA-API entry
point (src/vaapi/vaapi_entrypoint.c:457-471) and frames in submission order.

The harness is built where the reference tree exists (make -C integration,
run by the build) and travels with the tree."""
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "integration", "_build", "dropin_harness")


@pytest.mark.parametrize("size", [(352, 288), (1280, 720), (1920, 1080)])
def test_reference_api_decodes_through_cuda(size):
    if not os.path.exists(HARNESS):
        pytest.fail("integration/_build/dropin_harness is not built (make -C integration where the "
                    "reference tree is present)")
    w, h = size
    p = subprocess.run([HARNESS, str(w), str(h), "24", "10"], capture_output=True, text=True, timeout=300)
    line = [x for x in p.stdout.splitlines() if x.startswith("{")]
    assert line, p.stdout + p.stderr
    r = json.loads(line[-1])
    assert r["cuda_active"] == 1, p.stderr
    assert r["errors"] == 0 and r["out_of_order"] == 0, r
    assert r["compared"] == 24 and r["mismatched"] == 0, r
    assert r["again"] > 0, r              # the ring filled and the caller drained it
    assert p.returncode == 0
