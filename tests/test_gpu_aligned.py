"""Restart-aligned graph runs of the batched Lanczos.

``LanczosBatch.run_aligned`` replays a head graph of ``keep`` steps and then
cycles of ``n_slots - keep`` steps that launch the Ritz check and the thick
restart after their last step only.  It issues the kernels of
``run(graph=True)`` in the same order minus the Ritz launches that find no
check due, so eigenvalues, residuals and the per-instance iteration and
restart counts must agree bit for bit.
"""

import numpy as np
import pytest

from _cases import ed_data_for

pytestmark = pytest.mark.gpu


def _pair(case, golden, prec, **kw):
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200.lanczos import LanczosBatch

    g = golden(case)
    data = ed_data_for(case, g)
    dm, sset = data._device()
    sectors = [int(s) for s in g["eig_sectors"]]
    nev = int(g["nev"])
    p = ed.LanczosParams(precision=prec, **kw)
    return g, sectors, nev, (LanczosBatch(dm, sset, sectors, nev, p), LanczosBatch(dm, sset, sectors, nev, p))


def _solve(b, aligned):
    b.load_start(None)
    b.start()
    st = b.run_aligned(poll=16) if aligned else b.run(poll=16, graph=True)
    return st, b.ritz_val[:, : b.nev].cpu().numpy(), b.resid[:, : b.nev].cpu().numpy()


@pytest.mark.parametrize("case,prec", [("checkerboard24", 32), ("checkerboard24", 64), ("haldane24_flux", 64),
                                       ("heisenberg16", 64)])
def test_aligned_matches_per_poll_graph(golden, case, prec):
    from realspace_exatdiagonalization_py_b200.lanczos import S_ITERS, S_NCONV, S_RESTARTS, S_STATUS

    g, sectors, nev, (a, b) = _pair(case, golden, prec)
    assert a.restart_period == a.p.n_slots - a.keep
    for rep in range(2):  # the second solve replays the head graph instead of the eager head
        st_a, va, ra = _solve(a, True)
        st_b, vb, rb = _solve(b, False)
        np.testing.assert_array_equal(va, vb)
        np.testing.assert_array_equal(ra, rb)
        for col in (S_ITERS, S_RESTARTS, S_STATUS, S_NCONV):
            np.testing.assert_array_equal(st_a[:, col], st_b[:, col])
        # every instance converged at the check of a restart step: n_slots
        # steps after start, then every restart_period steps
        assert np.all(st_a[:, S_STATUS] == 1)
        steps = st_a[:, S_ITERS] - 1
        np.testing.assert_array_equal(steps, a.keep + (st_a[:, S_RESTARTS] + 1) * a.restart_period)
    assert a.replayed_launches > 0
    if prec == 64:
        for i, s in enumerate(sectors):
            ref = g["eig_vals"][list(g["eig_sectors"]).index(s)]
            m = min(nev, len(ref))
            np.testing.assert_allclose(va[i, :m], ref[:m], atol=1e-10, rtol=0)


def test_periodic_check_inside_a_cycle_falls_back(golden):
    """check_every = 20 falls inside the second cycle: the rest of the solve
    takes the per-step path, with the same results as the per-poll graph."""
    from realspace_exatdiagonalization_py_b200.lanczos import S_ITERS, S_RESTARTS, S_STATUS

    _, _, _, (a, b) = _pair("checkerboard24", golden, 64, check_every=20)
    st_a, va, _ = _solve(a, True)
    st_b, vb, _ = _solve(b, False)
    np.testing.assert_array_equal(va, vb)
    for col in (S_ITERS, S_RESTARTS, S_STATUS):
        np.testing.assert_array_equal(st_a[:, col], st_b[:, col])


def test_span_past_a_due_restart_is_an_error(golden):
    """A span without Ritz launches that runs past the full basis stops every
    instance with RSED_EINVAL at the next Gram pass (nothing is written past
    the basis slots)."""
    from realspace_exatdiagonalization_py_b200 import _lib
    from realspace_exatdiagonalization_py_b200.lanczos import S_ACTIVE, S_STATUS

    _, _, _, (a, _) = _pair("checkerboard24", golden, 64)
    a.load_start(None)
    a.start()
    a.iterate_span(a.p.n_slots + 1, ritz_last=False)
    st = a.status()
    assert np.all(st[:, S_STATUS] == _lib.RSED_EINVAL)
    assert not st[:, S_ACTIVE].any()
    with pytest.raises(_lib.RsedError):
        a._final_status()
