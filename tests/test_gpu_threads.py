"""Entry points called on one context from several host threads, each with its own stream
(the drop-in contract of the Rayon callers): the per-context guard serialises the calls, so
every result equals the serial one bit for bit, for device-buffer calls on separate streams and
for host-buffer calls, with the m = 0 and m > 0 evaluators both in the batches."""
import threading

import numpy as np
import pytest

import nociwick
from nociwick import synthetic as sy

pytestmark = pytest.mark.gpu


def test_concurrent_calls_on_one_context_match_serial():
    import torch
    system = sy.make_system(12, 3, 3, 3, 24, seed=5, k_scale=0.3, zero_pairs=[(0, 1, 1, 0)], enuc=0.2)
    basis = sy.sd_basis(12, 3, 3, 3, orders=(1, 2, 3))
    batches = [sy.sample_pairs(basis, 200_000 + 1000 * k, seed=20 + k, distinct_parents=False).astype(np.uint32)
               for k in range(4)]
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-8).build() as w:
        w.set_basis(basis)
        serial = [w.eval_pairs(b) for b in batches]
        streams = [torch.cuda.Stream() for _ in batches]
        dps = [torch.from_numpy(b.view(np.int32)).cuda() for b in batches]
        outs = [torch.empty((b.shape[0], 2), dtype=torch.float64, device="cuda") for b in batches]
        host = [None] * len(batches)
        errors = []

        def device_worker(k):
            try:
                for _ in range(5):
                    outs[k].fill_(float("nan"))
                    w.eval_pairs_device(dps[k].data_ptr(), batches[k].shape[0], outs[k].data_ptr(),
                                        streams[k].cuda_stream)
                streams[k].synchronize()
            except Exception as e:  # reported below
                errors.append(e)

        def host_worker(k):
            try:
                for _ in range(3):
                    host[k] = w.eval_pairs(batches[k])
            except Exception as e:
                errors.append(e)

        threads = [threading.Thread(target=device_worker, args=(k,)) for k in range(len(batches))]
        threads += [threading.Thread(target=host_worker, args=(k,)) for k in range(len(batches))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        torch.cuda.synchronize()
    assert not errors, errors
    for k in range(len(batches)):
        assert np.array_equal(outs[k].cpu().numpy(), serial[k])
        assert np.array_equal(host[k], serial[k])
