"""Host-array calls move arrays of 16 MB and more through the pinned
staging ring (gpunufft_b200/csrc/hostcopy.cpp: 8 MB chunks, two buffers,
host threads filling one while the other's DMA runs).  The forward's
k-space output and the adjoint's k-space input here are 21.6 MB (two full
chunks and a partial one); the results must equal the device-array calls
on the same plan bit for bit, and a second round must give the same bits
again (the ring's buffers are reused)."""
import numpy as np
import pytest

from tests.helpers import cplx

pytestmark = pytest.mark.gpu


def test_staged_host_copies_equal_device_calls():
    torch = pytest.importorskip("torch")
    import gpunufft_b200 as G
    rng = np.random.default_rng(21)
    dims = (32, 32, 32)
    M, C = 100_000, 27  # 100,000 x 27 x 8 B = 21.6 MB of k-space
    traj = rng.uniform(-0.5, 0.5, (3, M)).astype(np.float32)
    p = G.Plan(traj, dims, 3, 8, 2.0, None, None, G.BALANCED)
    try:
        x = cplx(rng, C, *dims[::-1])
        k = cplx(rng, C, M)
        assert k.nbytes > 16 << 20 and k.nbytes % (8 << 20)
        for _ in range(2):
            y_host = p.forward(x)              # staged device -> host
            im_host = p.adjoint(k)             # staged host -> device
            y_dev = p.forward(torch.from_numpy(x).cuda()).cpu().numpy()
            im_dev = p.adjoint(torch.from_numpy(k).cuda()).cpu().numpy()
            assert np.array_equal(y_host.view(np.uint64), y_dev.view(np.uint64))
            assert np.array_equal(im_host.view(np.uint64),
                                  im_dev.view(np.uint64))
    finally:
        p.close()
