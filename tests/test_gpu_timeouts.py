"""The bounded waits' failure path, made to run out on purpose and safely: with the poll limit at
0 (cc_set_wait_limit), every mbarrier wait of the learned kernels (a CTA's wait for its own
tensor-core MMAs) gives up at once. Nothing is left hanging: the CTA first lets its committed MMAs
drain with the default limit, then frees its tensor memory, and the host reports
CC_DEVICE_TIMEOUT. With the default limit restored, the same kernels run again and give the normal
results bit for bit (a CTA that had kept its tensor memory would leave the next allocation short)."""
import numpy as np
import pytest
import torch

from helpers import cc, assert_cells_bitwise, bits

pytestmark = pytest.mark.gpu
_lib = __import__("cutcell_b200._lib", fromlist=["_lib"])
L = __import__("cutcell_b200.learned", fromlist=["learned"])


class wait_limit:
    def __init__(self, polls):
        self.polls = polls

    def __enter__(self):
        self.old = _lib.load().cc_set_wait_limit(self.polls)

    def __exit__(self, *a):
        _lib.load().cc_set_wait_limit(-1)


def test_learned_wait_timeout_frees_tensor_memory_and_recovers():
    rng = np.random.default_rng(1)
    X = torch.as_tensor(rng.uniform(-1.6, 1.6, (3000, 8)).astype(np.float32)).cuda()
    m = L.MLP(L.init_params(2))
    ref = m.predict(X).cpu().numpy()
    g = cc.workloads.unit_grid(64)
    body = cc.workloads.smooth_blob(3)
    plain = cc.update_cache(cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=torch.float32), body, g).to_host()
    learned = cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=torch.float32)
    with wait_limit(0):
        with pytest.raises(cc.CCError) as e:
            m.predict(X)
        assert e.value.status == _lib.CC_DEVICE_TIMEOUT
        with pytest.raises(cc.CCError) as e:
            L.update_cache_learned(learned, body, g, m, bound=-1.0)
        assert e.value.status == _lib.CC_DEVICE_TIMEOUT
    # every CTA released its tensor memory: the same kernels allocate it again and agree bit for bit
    assert np.array_equal(bits(m.predict(X).cpu().numpy()), bits(ref))
    L.update_cache_learned(learned, body, g, m, bound=-1.0)  # rejects every correction: the plain update
    assert_cells_bitwise(learned.to_host(), plain, label="learned update after a timeout")
