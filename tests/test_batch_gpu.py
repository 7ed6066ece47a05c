"""GPU parity of the batched per-target searches: all 4096 uneven instances of
the batch workload against the reference's per-instance checksums, under each
method policy, plus the device path (plan + CUDA graph replay)."""

import os

import numpy as np
import pytest

from bmmpy_b200 import batch as B
from bmmpy_b200.workloads import C4, batch_instance
from tests.golden.fixtures import checksum_pairs

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def wl():
    return np.load(os.path.join(GOLDEN, "workloads.npz"))


@pytest.fixture(scope="module")
def c4_batch():
    insts = [batch_instance(i) for i in range(C4["count"])]
    return B.Batch([(m, k) for m, k, _ in insts])


@pytest.fixture(autouse=True)
def _policy():
    B.set_policy(4, -1)
    yield
    B.set_policy(4, -1)


@pytest.mark.parametrize("gray_words,force", [(4, -1), (0, 0), (8, 2)])
def test_all_c4_instances_match_reference(wl, c4_batch, gray_words, force):
    B.set_policy(gray_words, force)
    masks, weights = c4_batch.run()
    first = wl["c4_first32"]
    assert np.array_equal(masks[: len(first)], first[:, 0])
    assert np.array_equal(weights[: len(first)].astype(np.uint64), first[:, 1])
    bad = [i for i, (m, w) in enumerate(zip(c4_batch.split(masks), c4_batch.split(weights)))
           if checksum_pairs(m, w) != int(wl["c4_checksums"][i])]
    assert bad == []


def test_c4_device_path_graph_replay(wl, c4_batch):
    import torch

    dev = torch.device("cuda", 0)
    dw = torch.from_numpy(c4_batch.words.view(np.int64).copy()).to(dev)
    dm = torch.full((c4_batch.n_out,), -1, dtype=torch.int64, device=dev)
    dwt = torch.full((c4_batch.n_out,), -1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    info = c4_batch.info()
    assert info["items"] == c4_batch.n_out and info["gray"] + info["fwht16"] + info["fwht_small"] > 0
    for _ in range(3):  # the second and third runs replay the captured graph
        c4_batch.run_dev(dw, dm, dwt, stream)
    torch.cuda.synchronize()
    masks = dm.cpu().numpy().view(np.uint64)
    weights = dwt.cpu().numpy().view(np.uint32)
    for i in (0, 1, 2, 1000, 4095):
        assert checksum_pairs(c4_batch.split(masks)[i],
                              c4_batch.split(weights)[i]) == int(wl["c4_checksums"][i])
    c4_batch.close()


def test_batch_rejects_bad_instances():
    from bmmpy_b200.workloads import gen_instance

    m, _ = gen_instance(5, 64, 0.3, 1)
    with pytest.raises(ValueError):
        B.Batch([(m, 5)]).run()  # k must be < rows
    m, _ = gen_instance(20, 40000, 0.3, 1)
    with pytest.raises(ValueError):
        B.Batch([(m, 16)]).run()  # too wide for both methods
