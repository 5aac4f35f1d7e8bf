"""The thick restart (``rsed_lanczos_restart``: the whole-row kernel and the
per-instance kernel) against numpy on random data: for every instance with
S_RESTART_NB = nb_old > 0,

    V_new[:, j] = sum_{l < (nb_old - 1) b} V[:, l] S[l, j]   (j < keep b)

(column l of the old basis = slot l // b, column c0 + l % b) and the residual
block (slot nb_old - 1) moved to slot keep; instances with nb_old = 0 and
columns outside the batch keep their values.  Tolerance 1e-12 relative to
the column norms (FP64 sums in a different order).
"""

import numpy as np
import pytest
import torch

from _cases import ed_data_for

pytestmark = pytest.mark.gpu


def _expected(V, S, nb_old, keep, bs, c0s):
    out = V.copy()
    for i, (nbo, b, c0) in enumerate(zip(nb_old, bs, c0s)):
        if nbo == 0:
            continue
        M, K = (nbo - 1) * b, keep * b
        Vi = np.stack([V[l // b, :, c0 + l % b] for l in range(M)], axis=1)  # [n, M]
        new = Vi @ S[i, :M, :K]
        for j in range(K):
            out[j // b, :, c0 + j % b] = new[:, j]
        out[keep, :, c0:c0 + b] = V[nbo - 1, :, c0:c0 + b]
    return out


@pytest.mark.parametrize("case,bs", [("checkerboard24", [4]), ("heisenberg16", [2]), ("heisenberg16", [1, 2, 3])])
@pytest.mark.parametrize("row_restart", [True, False])
def test_restart_matches_numpy(golden, case, bs, row_restart):
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200.lanczos import S_RESTART_NB, LanczosBatch

    g = golden(case)
    data = ed_data_for(case, g)
    dm, sset = data._device()
    sectors = [int(s) for s in g["eig_sectors"]]
    block_sizes = [bs[i % len(bs)] for i in range(len(sectors))]
    p = ed.LanczosParams(block=max(block_sizes), precision=64, row_restart=row_restart)
    b = LanczosBatch(dm, sset, sectors, int(g["nev"]), p, block_sizes=block_sizes)
    rng = np.random.default_rng(7)
    V0 = rng.standard_normal(b.V.shape) + 1j * rng.standard_normal(b.V.shape)
    S = rng.standard_normal(b.ritz_vec.shape) + 1j * rng.standard_normal(b.ritz_vec.shape)
    n_slots = p.n_slots
    # a restart normally comes with n_slots + 1 blocks (the last in the spare slot)
    nb_old = [n_slots + 1 if i % 4 else max(2, n_slots - i % 3) for i in range(len(sectors))]
    nb_old[1] = 0  # this instance does not restart
    b.V.copy_(torch.from_numpy(V0))
    b.ritz_vec.copy_(torch.from_numpy(S))
    st = b.state.cpu()
    st[:, S_RESTART_NB] = torch.tensor(nb_old, dtype=torch.int32)
    b.state.copy_(st)
    b.restart()
    torch.cuda.synchronize()
    got = b.V.cpu().numpy()
    c0s = b.inst_col0.cpu().numpy().tolist()
    want = _expected(V0, S, nb_old, b.keep, block_sizes, c0s)
    scale = np.abs(S).sum(axis=1).max() * np.abs(V0).max()
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12 * scale)
