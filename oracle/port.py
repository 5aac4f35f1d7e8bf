"""CPU restatement of the reference's symmetry-resolved ED path (numpy/scipy).

TEST INFRASTRUCTURE — the checker, never the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline/reference arm
import this module.  It restates, in vectorised numpy, the algorithm of
``src/realspace_exactdiagonalization_py/symmetry_resolved_ed.py`` (cited as
``SRE:line``):

* combinadic rank/unrank (SRE:122-140, 377-426),
* the two-pass chunked orbit-stabilizer sweep with byte lookup tables
  (SRE:346-374, 433-575) and its product-form edge case (SRE:483-508),
* ``update_orbit_stabilizer_phases`` (SRE:1220-1269),
* the sector filter (SRE:1484-1546),
* the per-term vectorised triplet builder (SRE:595-693) and the CSR operator
  (SRE:1913-1976),
* the sector-state -> Fock amplitude expansion
  (``observables/entanglement_spectrum.py:82-145``),
* the many-body Chern number on the flux torus: dictionary overlaps,
  determinant links and plaquette phases
  (``observables/many_body_chern_number.py:141-207, 341-438``),
* the charge pump: the orbit-diagonal position operator between sectors,
  manifold eigenvalues and phase-branch tracking
  (``observables/charge_pump.py:41-240, 325-505``),
* the one-body density matrix orbit by orbit as the reference computes it
  (``observables/off_diagonal_long_range_order.py:77-140``), and <a_i^dagger
  a_j>, <n_i n_j> as exact expectation values over the Fock amplitudes (the
  reference's <n_i n_j>, ``static_structure_factor.py:54-149``, is exactly
  that; its one-body density matrix equals it where alpha' conj(chi(g')) of
  every projected hop is real),
* the eigen-solves: dense ``eigh(UPLO="U")`` for n <= 500 and ARPACK
  ``eigs(k=nev, which="SR", tol=1e-10)`` with the seeded ``v0`` otherwise
  (SRE:2180-2299).

Its outputs are pinned against the reference engine itself (golden fixtures
in ``tests/golden/``, generated by ``tests/golden/make_golden.py`` through
``oracle/ref_shim.py``).  Unlike the reference it also ranks masks of more
than 42 sites correctly (the reference's fallback at SRE:665/896 passes
``n_site=0`` and returns rank 0 for every mask).
"""

from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def binom_table(n: int, k: int) -> np.ndarray:
    t = np.zeros((n + 1, k + 1), dtype=np.int64)
    for b in range(n + 1):
        for j in range(min(b, k) + 1):
            t[b, j] = math.comb(b, j)
    return t


def unrank(ranks: np.ndarray, n: int, k: int, bt: np.ndarray) -> np.ndarray:
    """SRE:377-394."""
    masks = np.zeros(len(ranks), dtype=np.uint64)
    r = ranks.astype(np.int64).copy()
    for j in range(k, 0, -1):
        b = np.minimum(np.searchsorted(bt[:, j], r, side="right") - 1, n - 1)
        masks |= np.uint64(1) << b.astype(np.uint64)
        r -= bt[b, j]
    return masks


def rank(masks: np.ndarray, n: int, bt: np.ndarray) -> np.ndarray:
    """Colex rank sum_j C(b_j, j+1), vectorised over masks (SRE:404-418 done
    with the real site count)."""
    masks = np.asarray(masks, dtype=np.uint64)
    out = np.zeros(masks.shape, dtype=np.int64)
    j = np.ones(masks.shape, dtype=np.int64)
    kmax = bt.shape[1] - 1
    for i in range(n):
        occ = ((masks >> np.uint64(i)) & np.uint64(1)).astype(bool)
        if occ.any():
            out[occ] += bt[i, np.minimum(j[occ], kmax)]
            j[occ] += 1
    return out


def species_basis(n: int, k: int, species, bt: np.ndarray):
    """(C, rank_fn, unrank_fn) of a basis.  ``species = (sb, kb)``: the sites
    in mask ``sb`` hold ``kb`` particles; rank = rank_A * C(|B|, kb) + rank_B,
    each species in colex order over its own sites (the device convention;
    the reference ranks one species only, SRE:122-140)."""
    if not species:
        return math.comb(n, k), (lambda m: rank(m, n, bt)), (lambda r: unrank(r, n, k, bt))
    sb, kb = species
    sites_b = [i for i in range(n) if (sb >> i) & 1]
    sites_a = [i for i in range(n) if not (sb >> i) & 1]
    na, nb, ka = len(sites_a), len(sites_b), k - kb
    cb = math.comb(nb, kb)

    def compact(m, sites):
        m = np.asarray(m, dtype=np.uint64)
        out = np.zeros(m.shape, dtype=np.uint64)
        for p, st in enumerate(sites):
            out |= ((m >> np.uint64(st)) & np.uint64(1)) << np.uint64(p)
        return out

    def deposit(cm, sites):
        out = np.zeros(cm.shape, dtype=np.uint64)
        for p, st in enumerate(sites):
            out |= ((cm >> np.uint64(p)) & np.uint64(1)) << np.uint64(st)
        return out

    def rank2(m):
        return rank(compact(m, sites_a), na, bt) * cb + rank(compact(m, sites_b), nb, bt)

    def unrank2(r):
        r = np.asarray(r, dtype=np.int64)
        return deposit(unrank(r // cb, na, ka, bt), sites_a) | deposit(unrank(r % cb, nb, kb, bt), sites_b)

    return math.comb(na, ka) * cb, rank2, unrank2


def _byte_tables(n: int, perm0: np.ndarray, angle: np.ndarray):
    """Per (g, byte, value): image bits and the byte's angle partial sum,
    bits ascending (SRE:346-374)."""
    ng = perm0.shape[0]
    nbytes = (n + 7) // 8
    ptab = np.zeros((ng, nbytes, 256), dtype=np.uint64)
    atab = np.zeros((ng, nbytes, 256), dtype=np.float64)
    for g in range(ng):
        for b in range(nbytes):
            for v in range(256):
                out, ang = 0, 0.0
                for i in range(8):
                    s = 8 * b + i
                    if s >= n:
                        break
                    if (v >> i) & 1:
                        out |= 1 << int(perm0[g, s])
                        ang += angle[g, s]
                ptab[g, b, v] = out
                atab[g, b, v] = ang
    return ptab, atab, nbytes


def apply_product(m: int, perm0: np.ndarray, eta: np.ndarray, fermion: bool):
    """Product-form U_g on one mask (SRE:283-315 / 977-1008)."""
    new, ph, par = 0, complex(1.0), 1
    t = m
    while t:
        low = t & -t
        s = low.bit_length() - 1
        p = int(perm0[s]) + 1
        if fermion and (new >> p).bit_count() & 1:
            par = -par
        new |= 1 << (p - 1)
        ph *= eta[s]
        t ^= low
    return new, ph * par


def catalog(n: int, k: int, perm0: np.ndarray, eta: np.ndarray, fermion: bool, chunk: int = 1 << 16,
            species=None):
    """Orbit catalog: dict with reprs (uint64), stab_g (list of int arrays),
    stab_phase (list of complex128 arrays), rep_rank/rep_sym (int32),
    rep_amp (complex64) over all C(n, k) states (or the two-species basis of
    :func:`species_basis`)."""
    ng = perm0.shape[0]
    bt = binom_table(n, k)
    C, rank_fn, unrank_fn = species_basis(n, k, species, bt)
    rep_rank = np.full(C, -1, dtype=np.int32)
    rep_sym = np.zeros(C, dtype=np.int32)
    rep_amp = np.zeros(C, dtype=np.complex64)
    reprs, stab_g, stab_ph = [], [], []
    if k == 0 or k == n:  # SRE:483-508
        m = (1 << k) - 1
        gs, ps = [], []
        for g in range(ng):
            img, a = apply_product(m, perm0[g], eta[g], fermion)
            if img == m:
                gs.append(g)
                ps.append(a)
        reprs.append(m)
        stab_g.append(np.array(gs, dtype=np.int64))
        stab_ph.append(np.array(ps, dtype=np.complex128))
        for g in range(ng):
            img, a = apply_product(m, perm0[g], eta[g], fermion)
            idx = int(rank_fn(np.array([img], dtype=np.uint64))[0])
            rep_rank[idx] = 0
            rep_sym[idx] = g
            rep_amp[idx] = np.complex64(a)
        return dict(reprs=np.array(reprs, dtype=np.uint64), stab_g=stab_g, stab_phase=stab_ph,
                    rep_rank=rep_rank, rep_sym=rep_sym, rep_amp=rep_amp, binom=bt, rank=rank_fn)
    angle = np.angle(eta)
    ptab, atab, nbytes = _byte_tables(n, perm0, angle)
    inv = np.zeros((ng, n, n), dtype=np.int64)
    if fermion:
        for g in range(ng):
            for i in range(n):
                for j in range(i + 1, n):
                    if perm0[g, i] > perm0[g, j]:
                        inv[g, i, j] = 1
    for start in range(0, C, chunk):
        stop = min(start + chunk, C)
        masks = unrank_fn(np.arange(start, stop, dtype=np.int64))
        best = np.full(stop - start, np.iinfo(np.uint64).max, dtype=np.uint64)
        for g in range(ng):
            img = np.zeros(stop - start, dtype=np.uint64)
            for b in range(nbytes):
                img |= ptab[g, b][((masks >> np.uint64(8 * b)) & np.uint64(0xFF)).astype(np.int64)]
            best = np.minimum(best, img)
        pos = np.nonzero(best == masks)[0]
        if pos.size == 0:
            continue
        idx0 = len(reprs)
        rm = masks[pos]
        imgs = np.zeros((ng, pos.size), dtype=np.uint64)
        angs = np.zeros((ng, pos.size), dtype=np.float64)
        for g in range(ng):
            for b in range(nbytes):
                by = ((rm >> np.uint64(8 * b)) & np.uint64(0xFF)).astype(np.int64)
                imgs[g] |= ptab[g, b][by]
                angs[g] += atab[g, b][by]
        ph = np.exp(1j * angs)
        if fermion:
            bits = ((rm[:, None] >> np.arange(n, dtype=np.uint64)) & np.uint64(1)).astype(np.int64)
            for g in range(ng):
                ninv = (bits * (bits @ inv[g])).sum(axis=1)
                ph[g, (ninv & 1) == 1] *= -1.0 + 0.0j
        rk = rank_fn(imgs)
        ids = np.arange(idx0, idx0 + pos.size, dtype=np.int64)
        for g in range(ng):  # ascending g, last writer wins (SRE:556-560)
            rep_rank[rk[g]] = ids
            rep_sym[rk[g]] = g
            rep_amp[rk[g]] = ph[g].astype(np.complex64)
        fix = imgs == rm[None, :]
        for j in range(pos.size):
            gs = np.nonzero(fix[:, j])[0]
            reprs.append(int(rm[j]))
            stab_g.append(gs.astype(np.int64))
            stab_ph.append(ph[gs, j].astype(np.complex128))
    return dict(reprs=np.array(reprs, dtype=np.uint64), stab_g=stab_g, stab_phase=stab_ph,
                rep_rank=rep_rank, rep_sym=rep_sym, rep_amp=rep_amp, binom=bt, rank=rank_fn)


def _rank_of(cat: dict, masks, n: int):
    fn = cat.get("rank")
    return fn(masks) if fn is not None else rank(masks, n, cat["binom"])


def update_phases(cat: dict, n: int, perm0: np.ndarray, eta_new: np.ndarray, fermion: bool) -> dict:
    """In place, product form, ascending g (SRE:1220-1269)."""
    bt = cat["binom"]
    ng = perm0.shape[0]
    for o, m in enumerate(cat["reprs"]):
        m = int(m)
        for j, g in enumerate(cat["stab_g"][o]):
            cat["stab_phase"][o][j] = apply_product(m, perm0[g], eta_new[g], fermion)[1]
    for o, m in enumerate(cat["reprs"]):
        m = int(m)
        for g in range(ng):
            img, a = apply_product(m, perm0[g], eta_new[g], fermion)
            idx = int(_rank_of(cat, np.array([img], dtype=np.uint64), n)[0])
            if cat["rep_rank"][idx] == o:
                cat["rep_sym"][idx] = g
                cat["rep_amp"][idx] = np.complex64(a)
    return cat


def sector_orbits(cat: dict, chi: np.ndarray, atol: float = 1e-12) -> np.ndarray:
    """Orbits with |chi(h) - alpha_h| <= atol on the stabilizer (SRE:1484-1546)."""
    keep = []
    for o in range(len(cat["reprs"])):
        ok = True
        for g, a in zip(cat["stab_g"][o], cat["stab_phase"][o]):
            if not abs(chi[g] - a) <= atol:
                ok = False
                break
        if ok:
            keep.append(o)
    return np.array(keep, dtype=np.int64)


def triplets(cat: dict, n: int, orbits: np.ndarray, bilinear, density, chi, fermion: bool,
             include_diagonal: bool = True):
    """(rows, cols, vals, h_diag) of one sector block (SRE:595-693)."""
    reprs = cat["reprs"]
    rm = reprs[orbits]
    stab = np.array([len(cat["stab_g"][o]) for o in range(len(reprs))], dtype=np.int64)
    so = stab[orbits]
    bt = cat["binom"]
    in_basis = np.zeros(len(reprs), dtype=bool)
    in_basis[orbits] = True
    row_of = np.full(len(reprs), -1, dtype=np.int64)
    row_of[orbits] = np.arange(len(orbits))
    D = len(orbits)
    h_diag = np.zeros(D, dtype=np.complex128)
    for (i, j, v) in density:
        both = ((rm >> np.uint64(i - 1)) & np.uint64(1)).astype(bool) & (
            (rm >> np.uint64(j - 1)) & np.uint64(1)).astype(bool)
        h_diag[both] += complex(v)
    rows = [np.arange(D)] if include_diagonal else []
    cols = [np.arange(D)] if include_diagonal else []
    vals = [h_diag.copy()] if include_diagonal else []
    for (i, j, t) in bilinear:
        hop = np.uint64((1 << (i - 1)) | (1 << (j - 1)))
        frm = np.uint64(1 << (i - 1))
        c = np.nonzero((rm & hop) == frm)[0]
        if c.size == 0:
            continue
        idx = _rank_of(cat, rm[c] ^ hop, n)
        crep = cat["rep_rank"][idx]
        keep = np.nonzero(in_basis[crep])[0]
        if keep.size == 0:
            continue
        r = row_of[crep[keep]]
        cc = c[keep]
        g = cat["rep_sym"][idx[keep]]
        a = cat["rep_amp"][idx[keep]]
        hp = np.ones(keep.size, dtype=np.complex128)
        if fermion:
            lo, hi = min(i, j), max(i, j)
            between = ((1 << (hi - lo - 1)) - 1) << lo if hi - lo > 1 else 0
            flip = (np.bitwise_count(rm[cc] & np.uint64(between)) & 1) == 1
            hp[flip] = -1.0 + 0.0j
        el = complex(t) * hp * a * np.conj(chi[g]) * np.sqrt(so[r] / so[cc])
        rows.append(r)
        cols.append(cc)
        vals.append(el)
    return np.concatenate(rows), np.concatenate(cols), np.concatenate(vals), h_diag


def csr_block(cat, n, orbits, bilinear, density, chi, fermion) -> sp.csr_matrix:
    r, c, v, _ = triplets(cat, n, orbits, bilinear, density, chi, fermion, True)
    D = len(orbits)
    H = sp.coo_matrix((v, (r, c)), shape=(D, D)).tocsr()
    H.eliminate_zeros()
    return H


def solve(H: sp.csr_matrix, nev: int, seeded_v0: bool = True):
    """SRE:2248-2299 (matrix-free) / 2214-2245 (matrix mode, no v0)."""
    n = H.shape[0]
    if n == 0:
        return np.zeros(0), np.zeros((0, 0), dtype=np.complex128)
    if n <= 500:
        w, v = np.linalg.eigh(H.toarray(), UPLO="U")
        return w[:nev].real, v[:, :nev]
    v0 = None
    if seeded_v0:
        rng = np.random.default_rng(12345)
        v0 = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        v0 /= np.linalg.norm(v0)
    w, v = spla.eigs(H, k=nev, which="SR", v0=v0, tol=1e-10)
    o = np.argsort(w.real)
    return w.real[o], v[:, o]


def group_arrays(G):
    perm0 = np.array([[p - 1 for p in op.perm] for op in G.operations], dtype=np.uint8)
    eta = np.array([op.perm_phases for op in G.operations], dtype=np.complex128)
    return perm0, eta


def scan(model, n_filled: int, G, irreps, nev: int, sectors=None):
    """Full CPU scan: catalog + every requested sector (the reference's
    ``build_ed_data`` + ``ed_scan(mode="matrixfree")`` in one call).
    Returns ``{sector: (vals, dim)}``."""
    n = G.n_site
    fermion = model.particle_statistics.name == "FERMIONIC"
    perm0, eta = group_arrays(G)
    cat = catalog(n, n_filled, perm0, eta, fermion)
    out = {}
    for s in (range(len(irreps)) if sectors is None else sectors):
        chi = np.asarray(irreps[s].values, dtype=np.complex128)
        orbits = sector_orbits(cat, chi)
        H = csr_block(cat, n, orbits, model.bilinear_terms, model.density_density_terms, chi, fermion)
        w, _ = solve(H, nev)
        out[s] = (w, len(orbits))
    return out


def fock_expand(cat: dict, orbits: np.ndarray, c: np.ndarray, chi: np.ndarray, perm0: np.ndarray,
                eta: np.ndarray, fermion: bool, atol: float = 1e-12) -> dict:
    """Sector vector -> normalised Fock amplitudes {mask: amplitude}
    (observables/entanglement_spectrum.py:82-145): every representative with
    |c| > atol adds c / sqrt(|G| |Stab|) * conj(chi(g)) * U_g|s> for all g;
    amplitudes <= atol are dropped and the rest renormalised."""
    ng = perm0.shape[0]
    amps: dict = {}
    for col, o in enumerate(orbits):
        coeff = c[col]
        if abs(coeff) <= atol:
            continue
        pref = coeff / np.sqrt(ng * len(cat["stab_g"][o]))
        m = int(cat["reprs"][o])
        for g in range(ng):
            img, ph = apply_product(m, perm0[g], eta[g], fermion)
            amps[img] = amps.get(img, 0j) + pref * np.conj(chi[g]) * ph
    amps = {k: v for k, v in amps.items() if abs(v) > atol}
    norm2 = sum(abs(v) ** 2 for v in amps.values())
    if norm2 <= atol:
        raise ValueError("Expanded state has near-zero norm.")
    inv = 1.0 / np.sqrt(norm2)
    return {k: v * inv for k, v in amps.items()}


def fock_overlap(a: dict, b: dict) -> complex:
    """<a|b> of two {mask: amplitude} maps (many_body_chern_number.py:141-160)."""
    if len(a) <= len(b):
        return sum((np.conj(v) * b.get(k, 0j) for k, v in a.items()), 0j)
    return sum((np.conj(a.get(k, 0j)) * v for k, v in b.items()), 0j)


def chern(model, n_filled: int, labels, grid, nev: int, flux_setup, det_atol: float = 1e-10):
    """Many-body Chern number (many_body_chern_number.py:341-438) on the CPU.

    ``flux_setup(flux)`` moves ``model`` to the flux point and returns
    ``(G, irreps)``; ``labels`` is ``["identity"]`` or momentum tuples.  Each
    sector is solved in matrix mode (``solve(..., seeded_v0=False)``), its
    lowest ``nev`` states expanded with ``fock_expand``.  Returns a dict with
    ``chern_number``, ``berry_curvature``, ``link_det_abs_x/y``,
    ``energies[nx, ny, n]`` and ``n_singular`` (links replaced by 1)."""
    nx, ny = grid
    n = model.lattice.n_site
    fermion = model.particle_statistics.name == "FERMIONIC"
    states = [[None] * ny for _ in range(nx)]
    energies = np.zeros((nx, ny, len(labels) * nev))
    for ix in range(nx):
        for iy in range(ny):
            G, irreps = flux_setup([ix / nx, iy / ny])
            perm0, eta = group_arrays(G)
            cat = catalog(n, n_filled, perm0, eta, fermion)
            pts = []
            for label in labels:
                s = 0 if label == "identity" else next(i for i, ir in enumerate(irreps) if ir.label == label)
                chi = np.asarray(irreps[s].values, dtype=np.complex128)
                orbits = sector_orbits(cat, chi)
                H = csr_block(cat, n, orbits, model.bilinear_terms, model.density_density_terms, chi, fermion)
                w, v = solve(H, nev, seeded_v0=False)
                for lev in range(nev):
                    energies[ix, iy, len(pts)] = w[lev]
                    pts.append(fock_expand(cat, orbits, v[:, lev], chi, perm0, eta, fermion))
            states[ix][iy] = pts
    n_sing = 0

    def link(a, b):
        nonlocal n_sing
        M = np.array([[fock_overlap(x, y) for y in b] for x in a], dtype=np.complex128)
        z = np.linalg.det(M)
        if abs(z) <= det_atol:
            n_sing += 1
            return 1.0 + 0.0j, abs(z)
        return z / abs(z), abs(z)

    Ux = np.empty((nx, ny), dtype=np.complex128)
    Uy = np.empty((nx, ny), dtype=np.complex128)
    dx = np.empty((nx, ny))
    dy = np.empty((nx, ny))
    for ix in range(nx):
        for iy in range(ny):
            Ux[ix, iy], dx[ix, iy] = link(states[ix][iy], states[(ix + 1) % nx][iy])
            Uy[ix, iy], dy[ix, iy] = link(states[ix][iy], states[ix][(iy + 1) % ny])
    F = np.empty((nx, ny))
    for ix in range(nx):
        for iy in range(ny):
            ixp, iyp = (ix + 1) % nx, (iy + 1) % ny
            F[ix, iy] = np.angle(Ux[ix, iy] * Uy[ixp, iy] * np.conj(Ux[ix, iyp]) * np.conj(Uy[ix, iy]))
    return {"chern_number": float(F.sum()) / (2 * np.pi), "berry_curvature": F, "link_det_abs_x": dx,
            "link_det_abs_y": dy, "energies": energies, "n_singular": n_sing}


def position_element(m: int, perm0: np.ndarray, w: np.ndarray, site_phase: np.ndarray) -> complex:
    """(1/|G|) sum_g w_g z(g(m)), z = product of site phases over the occupied
    sites in ascending order; |elem| <= 1e-13 -> 0 (charge_pump.py:102-161)."""
    ng = perm0.shape[0]
    e = 0j
    for g in range(ng):
        img = 0
        for i in range(perm0.shape[1]):
            if (m >> i) & 1:
                img |= 1 << int(perm0[g, i])
        z = 1 + 0j
        for j in range(perm0.shape[1]):
            if (img >> j) & 1:
                z *= site_phase[j]
        e += w[g] * z
    e *= 1.0 / ng
    return e if abs(e) > 1e-13 else 0j


def _track(raw: np.ndarray) -> np.ndarray:
    """Branch tracking (charge_pump.py:180-240): exhaustive assignment with the
    least summed squared wrapped jump, first in lexicographic order."""
    import itertools

    out = np.empty_like(raw)
    out[0] = np.sort(raw[0])
    for t in range(1, raw.shape[0]):
        prev = out[t - 1]
        best, best_cost = None, np.inf
        for perm in itertools.permutations(range(raw.shape[1])):
            c = 0.0
            for d, j in enumerate(perm):
                x = raw[t, j] - prev[d]
                c += (x - round(x)) ** 2
            if c < best_cost:
                best, best_cost = perm, c
        for b, j in enumerate(best):
            out[t, b] = raw[t, j] + round(prev[b] - raw[t, j])
    return out


def charge_pump(model, n_filled: int, specs, thetas, flux_direction: int, site_phase: np.ndarray, flux_setup):
    """Charge pump (charge_pump.py:325-505) on the CPU.  ``specs`` = list of
    (sector label, 1-based level); ``flux_setup(flux)`` moves ``model`` to the
    flux point and returns ``(G, irreps)``.  Sectors solved in matrix mode
    with ``max(max level, 2)`` levels.  Returns ``(polarization_eigenvalues,
    polarizations, pumped_charges, energies)``."""
    n = model.lattice.n_site
    dim = model.lattice.dim
    fermion = model.particle_statistics.name == "FERMIONIC"
    labels = list(dict.fromkeys(lab for lab, _ in specs))
    need = {lab: max(lev for l2, lev in specs if l2 == lab) for lab in labels}
    nev = max(max(need.values()), 2)
    ev_all = np.zeros((len(thetas), len(specs)), dtype=np.complex128)
    energies = np.full((len(thetas), len(labels), max(need.values())), np.nan)
    for it, th in enumerate(thetas):
        flux = [0.0] * dim
        flux[flux_direction - 1] = float(th)
        G, irreps = flux_setup(flux)
        perm0, eta = group_arrays(G)
        cat = catalog(n, n_filled, perm0, eta, fermion)
        vecs, orbs, chis = {}, {}, {}
        for il, lab in enumerate(labels):
            s = next(i for i, ir in enumerate(irreps) if ir.label == lab)
            chi = np.asarray(irreps[s].values, dtype=np.complex128)
            o = sector_orbits(cat, chi)
            H = csr_block(cat, n, o, model.bilinear_terms, model.density_density_terms, chi, fermion)
            w, v = solve(H, nev, seeded_v0=False)
            energies[it, il, : need[lab]] = w[: need[lab]]
            vecs[lab], orbs[lab], chis[lab] = v, o, chi
        P = np.zeros((len(specs), len(specs)), dtype=np.complex128)
        for r, (lt, vt) in enumerate(specs):
            for c, (lf, vf) in enumerate(specs):
                w = chis[lt] * np.conj(chis[lf])
                pos_t = {int(o): k for k, o in enumerate(orbs[lt])}
                acc = 0j
                for k, o in enumerate(orbs[lf]):
                    kt = pos_t.get(int(o))
                    if kt is None:
                        continue
                    e = position_element(int(cat["reprs"][o]), perm0, w, site_phase)
                    acc += np.conj(vecs[lt][kt, vt - 1]) * e * vecs[lf][k, vf - 1]
                P[r, c] = acc
        ev = np.linalg.eigvals(P)
        ev_all[it] = ev[np.argsort(np.angle(ev))]
    pol = _track(np.angle(ev_all) / (2 * np.pi))
    return ev_all, pol, pol[-1] - pol[0], energies


def fock_correlators(amps: dict, n: int, fermion: bool):
    """``(rho, nn)`` of a normalised {mask: amplitude} state: rho[i, j] =
    <a_i^dagger a_j> (sign (-1)^(occupied sites strictly between i and j) for
    fermions) and nn[i, j] = <n_i n_j>, 0-based sites."""
    rho = np.zeros((n, n), dtype=np.complex128)
    nn = np.zeros((n, n))
    for m, a in amps.items():
        w = abs(a) ** 2
        occ = [i for i in range(n) if (m >> i) & 1]
        for i in occ:
            for j in occ:
                nn[i, j] += w
        for j in occ:
            rho[j, j] += w
            for i in range(n):
                if (m >> i) & 1:
                    continue
                m2 = m ^ (1 << j) ^ (1 << i)
                b = amps.get(m2)
                if b is None:
                    continue
                sign = 1.0
                if fermion:
                    lo, hi = min(i, j), max(i, j)
                    between = ((1 << (hi - lo - 1)) - 1) << (lo + 1) if hi - lo > 1 else 0
                    if bin(m & between).count("1") & 1:
                        sign = -1.0
                rho[i, j] += np.conj(b) * a * sign
    return rho, nn


def obdm_orbitwise(cat: dict, orbits: np.ndarray, c: np.ndarray, chi: np.ndarray, perm0: np.ndarray,
                   eta: np.ndarray, fermion: bool, n: int, k: int) -> np.ndarray:
    """rho[i, j] as off_diagonal_long_range_order.py:77-140 accumulates it:
    per representative and group element the ket c / sqrt(|G| |Stab|) *
    conj(chi(g)) * phase_g; |c|^2/|G| on the diagonal of every occupied site;
    for a hop j -> i onto an orbit of the sector the bra c_row *
    sqrt(|Stab_row| / |G|) * conj(alpha' conj(chi(g'))) from the catalog entry
    of the hopped mask, times the Jordan-Wigner sign of the hop."""
    bt = binom_table(n, k)
    pos = {int(o): t for t, o in enumerate(orbits)}
    ng = perm0.shape[0]
    rho = np.zeros((n, n), dtype=np.complex128)
    for t, o in enumerate(orbits):
        if c[t] == 0:
            continue
        s_mask = int(cat["reprs"][o])
        S = len(cat["stab_g"][o])
        for g in range(ng):
            km, ph = apply_product(s_mask, perm0[g], eta[g], fermion)
            ket = c[t] * ((1 / np.sqrt(ng) / np.sqrt(S)) * np.conj(chi[g]) * ph)
            for j in range(n):
                if not (km >> j) & 1:
                    continue
                rho[j, j] += abs(c[t]) ** 2 / ng
                for i in range(n):
                    if i == j or (km >> i) & 1:
                        continue
                    nm = km ^ (1 << j) ^ (1 << i)
                    r = int(rank(np.array([nm], dtype=np.uint64), n, bt)[0])
                    ro = int(cat["rep_rank"][r])
                    if ro not in pos:
                        continue
                    p = complex(cat["rep_amp"][r]) * np.conj(chi[int(cat["rep_sym"][r])])
                    bra = c[pos[ro]] * (np.sqrt(len(cat["stab_g"][ro])) / np.sqrt(ng) * np.conj(p))
                    sign = 1.0
                    if fermion:
                        lo, hi = min(i, j), max(i, j)
                        between = ((1 << (hi - lo - 1)) - 1) << (lo + 1) if hi - lo > 1 else 0
                        if bin(km & between).count("1") & 1:
                            sign = -1.0
                    rho[i, j] += np.conj(bra) * ket * sign
    return rho
