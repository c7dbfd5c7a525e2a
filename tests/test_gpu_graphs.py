"""CUDA-graph replay of repeated calls (cms_graph_enable): a replay equals a
fresh call, reads the current contents of the caller's buffers, and a call
with other buffers or sizes is captured anew."""
import numpy as np
import pytest

from conftest import assert_same
from oracle import oracle

pytestmark = pytest.mark.gpu


def _with_b(packed, b):
    from cudams.packing import PackedSpectra

    return PackedSpectra(packed.mz, packed.a, b, packed.offsets, packed.mz_power,
                         packed.intensity_power, packed.n_max_peaks)


def test_graph_replay_dense_and_sparse(cuda_device):
    import torch

    from cudams import _native, kernels, synthetic

    ctx = _native.context(cuda_device.index)
    ref = synthetic.uniform_spectra(200, seed=81)
    qry = synthetic.uniform_spectra(170, seed=82)
    rd, qd = ref.to_device(cuda_device), qry.to_device(cuda_device)
    out = tuple(torch.empty((200, 170), dtype=t, device=cuda_device)
                for t in (torch.float32, torch.int32, torch.uint8))
    cfg = {"mode": 1, "tile_spectra": 64}
    want = oracle.cosine_greedy(ref, qry, 0.1, 0.0, 2048)
    ctx.graph_enable(True)
    try:
        ctx.profile_read(reset=True)
        for rep in range(3):
            for t in out:
                t.fill_(7)
            got = kernels.cosine_greedy_dense(rd, qd, 0.1, 0.0, 2048, out=out, config=cfg,
                                              check_errors=True)
            assert_same(tuple(x.cpu().numpy() for x in got), want, f"replay {rep}")
        _, launches = ctx.profile_read(reset=True)
        assert launches.sum() >= 3 * 8  # every replay still counts its kernels

        # same pointers, new contents: the replay must read them
        rng = np.random.default_rng(83)
        b2 = ref.b.copy()
        idx = rng.integers(0, b2.shape[0], 500)
        b2[idx] = rng.random(500)
        rd.b.copy_(torch.from_numpy(b2))
        got = kernels.cosine_greedy_dense(rd, qd, 0.1, 0.0, 2048, out=out, config=cfg,
                                          check_errors=True)
        assert_same(tuple(x.cpu().numpy() for x in got),
                    oracle.cosine_greedy(_with_b(ref, b2), qry, 0.1, 0.0, 2048), "new contents")

        # other output buffers and another shape: captured anew
        out2 = tuple(t[:150] for t in (torch.empty((200, 170), dtype=x.dtype, device=cuda_device)
                                       for x in out))
        sub = ref.subset(0, 150)
        got = kernels.cosine_greedy_dense(_with_b(sub, b2[:sub.n_peaks]).to_device(cuda_device), qd,
                                          0.1, 0.0, 2048, out=out2, config=cfg, check_errors=True)
        assert_same(tuple(x.cpu().numpy() for x in got),
                    oracle.cosine_greedy(_with_b(sub, b2[:sub.n_peaks]), qry, 0.1, 0.0, 2048),
                    "other buffers")

        # sparse: the hit count is reset inside the graph on every replay
        full = oracle.cosine_greedy(_with_b(ref, b2), qry, 0.1, 0.0, 2048)
        thr = float(np.quantile(full[0], 0.9))
        wr, wq = np.nonzero(full[0] >= np.float32(thr))
        for rep in range(3):
            hits = kernels.cosine_greedy_sparse(rd, qd, 0.1, 0.0, 2048, thr, config=cfg,
                                                capacity=4 * wr.shape[0] + 16)
            r, q, sc, mt, ov = hits.to_host(sort=True)
            np.testing.assert_array_equal(r, wr)
            np.testing.assert_array_equal(q, wq)
            np.testing.assert_array_equal(sc.view(np.uint32), full[0][wr, wq].view(np.uint32))
    finally:
        ctx.graph_enable(False)
