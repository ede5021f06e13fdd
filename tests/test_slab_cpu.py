"""The slab decomposition of a field over several processes (mcstar_b200.slab), on CPU with
two and four gloo ranks: the all-to-all packing and the exchange move the carried field
between ky-slabs and z-slabs exactly as the decomposed step needs.  Each rank's local
passes (IFFT_z, the xy part with the cubic term, the z pass with the field's wavenumbers)
are the oracle's numpy transforms here, so the test checks the decomposition and the data
movement; after the steps the assembled half spectrum equals the oracle's step of the
whole field."""
import math
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


SHAPE, DX, DT, EPS, C, MU, STEPS = (12, 16, 8), math.pi / 4, 0.5, 0.3, 1.0, 0.02, 3


def _field():
    nx, ny, nz = SHAPE
    return -0.2 + 0.1 * np.random.default_rng(5).uniform(-1, 1, (nz, ny, nx))


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "mcstar-libs_b200"), os.path.join(root, "oracle")]
    import pfc_oracle as O
    from mcstar_b200 import dist
    from mcstar_b200 import slab as S
    dist.init("gloo", timeout_s=60)
    nx, ny, nz = SHAPE
    nys, nzs = ny // world, nz // world
    ky0 = rank * nys
    lens = (nx * DX, ny * DX, nz * DX)
    k2 = O.kgrid(SHAPE, lens)[:, ky0:ky0 + nys, :]
    kpsi = O.r2c(_field())[:, ky0:ky0 + nys, :]
    # the local passes as the library's slab entry points compute them
    A = np.fft.ifft(kpsi, axis=0)                                   # pfc_slab_zinv
    as_t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.float64).reshape(a.shape + (2,)))
    as_c = lambda t: t.numpy().view(np.complex128)[..., 0]
    for t in range(STEPS):
        Az = as_c(S.from_z_chunks(S.exchange(S.to_z_chunks(as_t(A), world))))
        psi = np.fft.irfft2(Az, s=(ny, nx), axes=(1, 2))            # pfc_slab_xy
        Bz = np.fft.rfft2(psi ** 3 - C * psi - MU, axes=(1, 2))
        B = as_c(S.from_ky_chunks(S.exchange(S.to_ky_chunks(as_t(Bz), world))))
        kp, kn = np.fft.fft(A, axis=0), np.fft.fft(B, axis=0)       # pfc_slab_zpass
        new = (kp - DT * k2 * kn) / (1.0 + DT * k2 * ((1.0 - k2) ** 2 + C - EPS))
        A = new if t == STEPS - 1 else np.fft.ifft(new, axis=0)
    q.put((rank, A))
    dist.shutdown(world)


@pytest.mark.parametrize("world", [2, 4])
def test_gloo_ranks_step_slabs_like_the_whole_field(world):
    import pfc_oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got = np.concatenate([res[r] for r in range(world)], axis=1)
    nx, ny, nz = SHAPE
    want = O.step(O.r2c(_field()), STEPS, DT, EPS, (nx * DX, ny * DX, nz * DX), SHAPE, mu=MU, C=C)
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-12


def test_packing_round_trips():
    from mcstar_b200 import slab as S
    g = 4
    a = torch.randn(8, 3, 5, 2)  # a ky-slab: NZ = 8 planes of 3 rows
    chunks = S.to_z_chunks(a, g)
    assert [c.shape[0] for c in chunks] == [2] * g
    assert torch.equal(S.from_ky_chunks(chunks), a)
    b = torch.randn(2, 12, 5, 2)  # a z-slab: 2 planes of NY = 12 rows
    assert torch.equal(S.from_z_chunks(S.to_ky_chunks(b, g)), b)
