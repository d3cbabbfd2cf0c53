"""Sim-file generator for the single-band Hubbard model on the square,
triangular, honeycomb and kagome lattices.

A restatement of the reference generator's create_1 / create_batch
(util/gen_1band_unified_hub.py:265-1200, with the periodic hopping
matrices and Peierls phases of util/tight_binding.py:4-432 and the RNG helpers of
util/gen_util_shared.py:5-66) that needs neither h5py nor git, so chains can
be generated wherever the engine runs.  It writes the datasets the engine
and the reference's sweep read -- the same names, dtypes, shapes and values
as the reference generator -- except the two-bond
family (bond2s, map_b2*, pp_*, used only by the thermal and two-bond
correlators) and the plaquette-pair maps, which are omitted.

make_sim(...) returns the datasets as a dict (no file); create_batch(...)
writes DQSF files like the reference (sim_i.h5 + an external-linked
prefix.h5.params).
"""
from __future__ import annotations

import os

import numpy as np
from scipy.linalg import expm

from . import simfile

GEN_ID = "dqmc-b200"

# ----------------------------------------------------------------- RNG
M64 = (1 << 64) - 1


def seed_splitmix64(x: int) -> np.ndarray:
    """gen_util_shared.py:12-21"""
    rng = np.zeros(17, dtype=np.uint64)
    x &= M64
    for i in range(16):
        x = (x + 0x9E3779B97F4A7C15) & M64
        z = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        rng[i] = z ^ (z >> 31)
    return rng


class Xorshift1024:
    """xorshift1024* over a 17-word state array (gen_util_shared.py:25-31)."""

    def __init__(self, state: np.ndarray):
        self.s = [int(v) for v in state[:16]]
        self.p = int(state[16])

    def next(self) -> int:
        s0 = self.s[self.p]
        self.p = (self.p + 1) & 15
        s1 = self.s[self.p]
        s1 ^= (s1 << 31) & M64
        self.s[self.p] = s1 ^ s0 ^ (s1 >> 11) ^ (s0 >> 30)
        return (self.s[self.p] * 1181783497276652981) & M64

    def state(self) -> np.ndarray:
        return np.array(self.s + [self.p], dtype=np.uint64)


_JUMP = (0x84242F96ECA9C41D, 0xA3C65B8776F96855, 0x5B34A39F070B5837, 0x4489AFFCE4F31A1E,
         0x2FFEEB0A48316F40, 0xDC2D9891FE68C022, 0x3659132BB12FEA70, 0xAAC17D8EFA43CAB8,
         0xC4CB815590989B13, 0x5EE975283D71C93B, 0x691548C86C1BD540, 0x7910C41D10A1E6A5,
         0x0B5FC64563B3E2A8, 0x047F7684E9FC949D, 0xB99181F2D8F685CA, 0x284600E3F30E38C3)


def rand_jump(rng: np.ndarray) -> np.ndarray:
    """2^512 steps ahead (gen_util_shared.py:34-66); returns the new state."""
    g = Xorshift1024(rng)
    t = [0] * 16
    for word in _JUMP:
        for b in range(64):
            if (word >> b) & 1:
                for j in range(16):
                    t[j] ^= g.s[(j + g.p) & 15]
            g.next()
    for j in range(16):
        g.s[(j + g.p) & 15] = t[j]
    return g.state()


def initial_hs(rng_state: np.ndarray, L: int, N: int):
    """hs[l, i] = rand_uint >> 63 in (l, i) order (gen_1band_unified_hub.py:325-328);
    returns the fields and the RNG state after the draws."""
    g = Xorshift1024(rng_state)
    hs = np.empty((L, N), dtype=np.int32)
    for l in range(L):
        for i in range(N):
            hs[l, i] = g.next() >> 63
    return hs, g.state()


# ----------------------------------------------------------- lattice
LATTICE = {
    # primitive vectors a1, a2 and the unit-cell area
    "square": (np.array((1, 0)), np.array((0, 1)), 1),
    "triangular": (np.array((0.5, np.sqrt(3) / 2)), np.array((-0.5, np.sqrt(3) / 2)),
                   np.sqrt(3) / 2),
}
NORB = {"square": 1, "triangular": 1, "honeycomb": 2, "kagome": 3}


def peierls(Nx: int, Ny: int, lattice: str, nflux: int, alpha: float = 0.5,
            r_to=np.array((0, 0)), r_from=np.array((0, 0))) -> np.ndarray:
    """Peierls phases exp(i p phi) of a uniform field B through the Nx x Ny
    torus of the Bravais lattice `lattice`, nflux flux quanta in all
    (p = 2 pi nflux / (area of the torus)).

    Gauge: A(r) = B (-alpha y, beta x), beta = 1 - alpha.  Hopping from the
    site at cell c_i + r_from to the site at cell c_j + r_to, with c_j = c_i
    + d for a displacement d in the central range, the straight-line
    integral of A is -alpha m_y d_x + beta m_x d_y (m the midpoint, d the
    displacement of the two positions).  When c_j lies outside the torus it
    is the wrapped cell c_j' = c_j - o, o = o1 a1 + o2 a2; the magnetic
    translation by o adds the gauge transform A_o . (r_j + r_j')/2 with
    A_o = (-alpha o_y, beta o_x), and the product o1 o2 (beta a2x a1y -
    alpha a1x a2y) that keeps the string of translations single-valued.
    Entry [j', i] = exp(i p (interior - (wrap + extra))).  The expression
    order is fixed: sim files written with these phases must equal the
    reference generator's bit for bit."""
    a1, a2, unit_area = LATTICE[lattice]
    beta = 1 - alpha
    pref = 2 * np.pi * nflux / (unit_area * Nx * Ny)
    phi = np.zeros((Ny * Nx, Ny * Nx))
    for dy in range((1 - Ny) // 2, (1 + Ny) // 2):
        for dx in range((1 - Nx) // 2, (1 + Nx) // 2):
            for iy in range(Ny):
                for ix in range(Nx):
                    jy, jx = iy + dy, ix + dx
                    jjy, jjx = jy % Ny, jx % Nx
                    o1, o2 = jx - jjx, jy - jjy
                    ri = ix * a1 + iy * a2 + r_from
                    rj = jx * a1 + jy * a2 + r_to
                    rjj = jjx * a1 + jjy * a2 + r_to
                    dr = rj - ri
                    mr = (ri + rj) / 2
                    a_off = np.array((-alpha * (o1 * a1[1] + o2 * a2[1]),
                                      beta * (o1 * a1[0] + o2 * a2[0])))
                    interior = -alpha * mr[1] * dr[0] + beta * mr[0] * dr[1]
                    wrap = np.dot(a_off, 0.5 * (rj + rjj))
                    extra = o1 * o2 * (beta * a2[0] * a1[1] - alpha * a1[0] * a2[1])
                    phi[jjx + Nx * jjy, ix + Nx * iy] = interior + (-1) * (wrap + extra)
    return np.exp(1j * pref * phi)


def peierls_square(Nx: int, Ny: int, nflux: int, alpha: float = 0.5) -> np.ndarray:
    """Peierls phases of the square lattice (see peierls)."""
    return peierls(Nx, Ny, "square", nflux, alpha)


def hopping_square(Nx: int, Ny: int, t: float = 1.0, tp: float = 0.0, nflux: int = 0):
    """Hopping matrix with periodic boundaries and its Peierls phases
    (H_periodic_square, util/tight_binding.py:81-136, no twist, no t'')."""
    N = Nx * Ny
    tij = np.zeros((N, N), dtype=np.complex128)
    for iy in range(Ny):
        for ix in range(Nx):
            iy1, ix1 = (iy + 1) % Ny, (ix + 1) % Nx
            tij[ix1 + Nx * iy, ix + Nx * iy] += -t
            tij[ix + Nx * iy, ix1 + Nx * iy] += -t
            tij[ix + Nx * iy1, ix + Nx * iy] += -t
            tij[ix + Nx * iy, ix + Nx * iy1] += -t
            tij[ix + Nx * iy, ix1 + Nx * iy1] += -tp
            tij[ix1 + Nx * iy1, ix + Nx * iy] += -tp
            tij[ix1 + Nx * iy, ix + Nx * iy1] += -tp
            tij[ix + Nx * iy1, ix1 + Nx * iy] += -tp
    ph = peierls_square(Nx, Ny, nflux)
    return tij * ph, ph


def hopping_triangular(Nx: int, Ny: int, t: float = 1.0, nflux: int = 0):
    """Nearest-neighbour hopping of the triangular lattice (a1 = (1/2,
    sqrt3/2), a2 = (-1/2, sqrt3/2): neighbours along x, y and x - y in cell
    indices) with periodic boundaries, and its Peierls phases
    (H_periodic_triangular, util/tight_binding.py:182-225)."""
    N = Nx * Ny
    tij = np.zeros((N, N), dtype=np.complex128)
    for iy in range(Ny):
        for ix in range(Nx):
            iy1, ix1 = (iy + 1) % Ny, (ix + 1) % Nx
            tij[ix1 + Nx * iy, ix + Nx * iy] += -t
            tij[ix + Nx * iy, ix1 + Nx * iy] += -t
            tij[ix + Nx * iy1, ix + Nx * iy] += -t
            tij[ix + Nx * iy, ix + Nx * iy1] += -t
            tij[ix1 + Nx * iy, ix + Nx * iy1] += -t
            tij[ix + Nx * iy1, ix1 + Nx * iy] += -t
    ph = peierls(Nx, Ny, "triangular", nflux)
    return tij * ph, ph


def hopping_honeycomb(Nx: int, Ny: int, t: float = 1.0, nflux: int = 0):
    """Honeycomb lattice: sublattice A (orbital 0) and B (orbital 1) on the
    triangular Bravais lattice, B at offset (0, -1/sqrt3) from A, each A
    bonded to the B of its own cell and of the cells +a1 (y) and +a2 (x)
    (H_periodic_honeycomb, util/tight_binding.py:228-325, t' = 0).  The
    A-A and B-B blocks take the Bravais phases, the A-B blocks the phases
    with the B offset."""
    C = Nx * Ny
    tij = np.zeros((2 * C, 2 * C), dtype=np.complex128)
    for iy in range(Ny):
        for ix in range(Nx):
            iy1, ix1 = (iy + 1) % Ny, (ix + 1) % Nx
            tij[ix + Nx * iy1 + C, ix + Nx * iy] += -t
            tij[ix1 + Nx * iy + C, ix + Nx * iy] += -t
            tij[ix + Nx * iy + C, ix + Nx * iy] += -t
            tij[ix + Nx * iy, ix + Nx * iy1 + C] += -t
            tij[ix + Nx * iy, ix1 + Nx * iy + C] += -t
            tij[ix + Nx * iy, ix + Nx * iy + C] += -t
    p_diag = peierls(Nx, Ny, "triangular", nflux)
    p_off = peierls(Nx, Ny, "triangular", nflux, r_to=np.array((0, -1 / np.sqrt(3))))
    K = tij.copy()
    P = np.full((2 * C, 2 * C), np.nan, dtype=np.complex128)
    P[:C, :C] = p_diag
    P[C:, C:] = p_diag
    P[:C, C:] = p_off.T.conj()
    P[C:, :C] = p_off
    K[:C, :C] *= p_diag
    K[C:, C:] *= p_diag
    K[:C, C:] *= p_off.T.conj()
    K[C:, :C] *= p_off
    return K, P


def hopping_kagome(Nx: int, Ny: int, t: float = 1.0, nflux: int = 0):
    """Kagome lattice: three sites per triangular cell, A (orbital 0) at the
    cell origin, B (1) at (1/4, -sqrt3/4) and C (2) at (-1/4, -sqrt3/4);
    bonds A-B within the cell and to the B of the cell +a1, A-C within the
    cell and to the A of the cell -a2, B-C within the cell and to the C of
    the cell +a2 -a1 (H_periodic_kagome, util/tight_binding.py:328-432,
    t' = 0).  Each block takes the phases of its two sublattice offsets."""
    C = Nx * Ny
    tij = np.zeros((3 * C, 3 * C), dtype=np.complex128)
    for iy in range(Ny):
        for ix in range(Nx):
            iy1, ix1 = (iy + 1) % Ny, (ix + 1) % Nx
            iyn1, ixn1 = (iy - 1) % Ny, (ix - 1) % Nx
            tij[ix + Nx * iy1 + C, ix + Nx * iy] += -t
            tij[ix + Nx * iy + C, ix + Nx * iy] += -t
            tij[ix + Nx * iy, ix + Nx * iy1 + C] += -t
            tij[ix + Nx * iy, ix + Nx * iy + C] += -t
            tij[ixn1 + Nx * iy, ix + Nx * iy + 2 * C] += -t
            tij[ix + Nx * iy, ix + Nx * iy + 2 * C] += -t
            tij[ix + Nx * iy + 2 * C, ixn1 + Nx * iy] += -t
            tij[ix + Nx * iy + 2 * C, ix + Nx * iy] += -t
            tij[ix1 + Nx * iyn1 + 2 * C, ix + Nx * iy + C] += -t
            tij[ix + Nx * iy + 2 * C, ix + Nx * iy + C] += -t
            tij[ix + Nx * iy + C, ix1 + Nx * iyn1 + 2 * C] += -t
            tij[ix + Nx * iy + C, ix + Nx * iy + 2 * C] += -t
    off_b = np.array((1 / 4, -np.sqrt(3) / 4))
    off_c = np.array((-1 / 4, -np.sqrt(3) / 4))
    p_01 = peierls(Nx, Ny, "triangular", nflux, r_to=off_b, r_from=np.array((0, 0)))
    p_20 = peierls(Nx, Ny, "triangular", nflux, r_to=0, r_from=off_c)
    p_12 = peierls(Nx, Ny, "triangular", nflux, r_to=off_c, r_from=off_b)
    K = tij.copy()
    P = np.full((3 * C, 3 * C), np.nan, dtype=np.complex128)
    p_diag = peierls(Nx, Ny, "triangular", nflux)
    P[0:C, 0:C] = p_diag
    P[C:2 * C, C:2 * C] = p_diag
    P[2 * C:3 * C, 2 * C:3 * C] = p_diag
    P[0:C, C:2 * C] = p_01.T.conj()
    P[C:2 * C, 0:C] = p_01
    P[2 * C:3 * C, 0:C] = p_20.T.conj()
    P[0:C, 2 * C:3 * C] = p_20
    P[2 * C:3 * C, C:2 * C] = p_12
    P[C:2 * C, 2 * C:3 * C] = p_12.T.conj()
    K[C:2 * C, 0:C] *= p_01
    K[0:C, C:2 * C] *= p_01.T.conj()
    K[2 * C:3 * C, 0:C] *= p_20.T.conj()
    K[0:C, 2 * C:3 * C] *= p_20
    K[2 * C:3 * C, C:2 * C] *= p_12
    K[C:2 * C, 2 * C:3 * C] *= p_12.T.conj()
    return K, P


def square_maps(Nx: int, Ny: int, tp: float):
    """Measurement maps of the square lattice with translation symmetry
    (gen_1band_unified_hub.py:44-200, 420-520)."""
    N = Nx * Ny
    bps = 4 if tp != 0.0 else 2
    b2ps = 12 if tp != 0.0 else 4
    m = {}
    m["map_i"] = np.zeros(N, dtype=np.int32)
    m["num_i"], m["degen_i"] = 1, N
    map_ij = np.zeros((N, N), dtype=np.int32)
    for jy in range(Ny):
        for jx in range(Nx):
            for iy in range(Ny):
                for ix in range(Nx):
                    map_ij[jx + Nx * jy, ix + Nx * iy] = (ix - jx) % Nx + Nx * ((iy - jy) % Ny)
    m["map_ij"], m["num_ij"], m["degen_ij"] = map_ij, N, N
    bonds = np.zeros((2, bps * N), dtype=np.int32)
    for iy in range(Ny):
        for ix in range(Nx):
            i = ix + Nx * iy
            iy1, ix1 = (iy + 1) % Ny, (ix + 1) % Nx
            bonds[:, i] = (i, ix1 + Nx * iy)
            bonds[:, i + N] = (i, ix + Nx * iy1)
            if bps == 4:
                bonds[:, i + 2 * N] = (i, ix1 + Nx * iy1)
                bonds[:, i + 3 * N] = (ix1 + Nx * iy, ix + Nx * iy1)
    m["bonds"], m["num_b"], m["bps"], m["b2ps"] = bonds, bps * N, bps, b2ps
    m["map_b"] = np.tile(np.arange(bps, dtype=np.int32), (N, 1)).T.flatten()
    m["num_b_accum"], m["degen_b"] = bps, N
    map_bs = np.zeros((N, bps * N), dtype=np.int32)
    map_bb = np.zeros((bps * N, bps * N), dtype=np.int32)
    for j in range(N):
        for i in range(N):
            k = map_ij[j, i]
            for ib in range(bps):
                map_bs[j, i + N * ib] = k + N * ib
            for jb in range(bps):
                for ib in range(bps):
                    map_bb[j + N * jb, i + N * ib] = k + N * (ib + bps * jb)
    m["map_bs"], m["num_bs"], m["degen_bs"] = map_bs, bps * N, N
    m["map_bb"], m["num_bb"], m["degen_bb"] = map_bb, bps * bps * N, N
    # plaquettes (gen_1band_unified_hub.py:44-99)
    plaqs = np.zeros((3, 2 * N), dtype=np.int32)
    for iy in range(Ny):
        for ix in range(Nx):
            i = ix + Nx * iy
            iy1, ix1 = (iy + 1) % Ny, (ix + 1) % Nx
            plaqs[:, i] = (i, ix1 + Nx * iy, ix + Nx * iy1)
            plaqs[:, i + N] = (ix1 + Nx * iy, ix1 + Nx * iy1, ix + Nx * iy1)
    m["plaqs"] = plaqs
    m["map_plaq"] = np.repeat(np.arange(2, dtype=np.int32), N)
    m["num_plaq"], m["num_plaq_accum"], m["degen_plaq"] = 2 * N, 2, N
    m["plaq_per_cell"] = 2
    # sizes of the two-bond family (its maps are not written)
    m["num_b2"], m["num_b2_accum"], m["degen_b2"] = b2ps * N, b2ps, N
    m["num_b2b2"], m["num_bb2"], m["num_b2b"] = b2ps * b2ps * N, bps * b2ps * N, b2ps * bps * N
    m["degen_bb2"] = m["degen_b2b"] = m["degen_b2b2"] = N
    return m


def orbital_maps(geometry: str, Nx: int, Ny: int, tp: float):
    """Measurement maps of the triangular, honeycomb and kagome lattices with
    translation symmetry, as the reference generator writes them
    (gen_1band_unified_hub.py:44-260, 694-895): per-orbital site classes,
    pair classes by displacement and the two orbitals, the plaquettes of the
    triangular and kagome lattices.  The bond, bond-site and bond-bond maps
    of these lattices are placeholders there (bonds and maps all zero,
    degeneracies zero), and are the same placeholders here."""
    if tp != 0.0:
        raise NotImplementedError("t' on the triangular, honeycomb and kagome lattices")
    norb = NORB[geometry]
    C = Nx * Ny
    N = norb * C
    bps = {"triangular": 3, "honeycomb": 3, "kagome": 4}[geometry]
    b2ps = 4
    m = {}
    m["map_i"] = np.repeat(np.arange(norb, dtype=np.int32), C)
    m["num_i"], m["degen_i"] = norb, C
    map_ij = np.zeros((N, N), dtype=np.int32)
    for jo in range(norb):
        for jy in range(Ny):
            for jx in range(Nx):
                for io in range(norb):
                    for iy in range(Ny):
                        for ix in range(Nx):
                            k = (ix - jx) % Nx + Nx * ((iy - jy) % Ny) + C * io + C * norb * jo
                            map_ij[jx + Nx * jy + C * jo, ix + Nx * iy + C * io] = k
    m["map_ij"], m["num_ij"], m["degen_ij"] = map_ij, norb * norb * C, C
    m["bonds"], m["num_b"], m["bps"], m["b2ps"] = (np.zeros((2, bps * N), dtype=np.int32),
                                                   bps * N, bps, b2ps)
    m["map_b"] = np.tile(np.arange(bps, dtype=np.int32), (N, 1)).T.flatten()
    m["num_b_accum"], m["degen_b"] = bps, N
    m["map_bs"], m["num_bs"], m["degen_bs"] = np.zeros((N, bps * N), dtype=np.int32), bps * N, 0
    m["map_bb"], m["num_bb"], m["degen_bb"] = (np.zeros((bps * N, bps * N), dtype=np.int32),
                                               bps * bps * N, 0)
    ppc = 1 if geometry == "honeycomb" else 2
    plaqs = np.zeros((3, ppc * C), dtype=np.int32)
    for iy in range(Ny):
        for ix in range(Nx):
            i = ix + Nx * iy
            iy1, ix1 = (iy + 1) % Ny, (ix + 1) % Nx
            if geometry == "triangular":
                plaqs[:, i] = (i, ix1 + Nx * iy, ix + Nx * iy1)
                plaqs[:, i + C] = (ix1 + Nx * iy, ix1 + Nx * iy1, ix + Nx * iy1)
            elif geometry == "kagome":
                plaqs[:, i] = (i, i + 2 * C, i + C)
                plaqs[:, i + C] = (i, ix1 + Nx * iy + 2 * C, ix + Nx * iy1 + C)
    m["plaqs"] = plaqs
    m["map_plaq"] = np.repeat(np.arange(ppc, dtype=np.int32), C)
    m["num_plaq"], m["num_plaq_accum"], m["degen_plaq"] = ppc * C, ppc, C
    m["plaq_per_cell"] = ppc
    m["num_b2"], m["num_b2_accum"], m["degen_b2"] = b2ps * N, b2ps, N
    m["num_b2b2"], m["num_bb2"], m["num_b2b"] = b2ps * b2ps * N, bps * b2ps * N, b2ps * bps * N
    m["degen_bb2"] = m["degen_b2b"] = m["degen_b2b2"] = 0
    return m


# ---------------------------------------------------------------- files
def make_sim(Nx=4, Ny=4, mu=0.0, tp=0.0, U=6.0, dt=0.1, L=40, nflux=0, h=0.0,
             n_delay=16, n_matmul=8, n_sweep_warm=200, n_sweep_meas=2000, period_eqlt=8,
             period_uneqlt=0, checkpoint_every=10000, meas_bond_corr=0, seed=None,
             init_rng=None, geometry="square") -> dict:
    """All datasets of one sim file (create_1,
    gen_1band_unified_hub.py:265-1160) as a dict name -> array, for the
    square, triangular, honeycomb or kagome lattice (periodic boundaries;
    t' on the square lattice only, as the reference generator)."""
    assert L % n_matmul == 0 and L % period_eqlt == 0
    if geometry not in NORB:
        raise NotImplementedError(f"geometry {geometry}")
    cplx = nflux != 0
    nt = np.complex128 if cplx else np.float64
    if init_rng is None:
        init_rng = seed_splitmix64(0 if seed is None else seed)
    N = NORB[geometry] * Nx * Ny
    hs, rng = initial_hs(init_rng, L, N)
    if geometry == "square":
        m = square_maps(Nx, Ny, tp)
        K, ph = hopping_square(Nx, Ny, 1.0, tp, nflux)
    else:
        m = orbital_maps(geometry, Nx, Ny, tp)
        K, ph = {"triangular": hopping_triangular, "honeycomb": hopping_honeycomb,
                 "kagome": hopping_kagome}[geometry](Nx, Ny, 1.0, nflux)
    if not cplx:
        K, ph = K.real, ph.real
    Ku = K.copy()
    Kd = K.copy()
    for i in range(N):
        Ku[i, i] -= mu - h
        Kd[i, i] -= mu + h
    U_i = U * np.ones(m["num_i"], dtype=np.float64)
    exp_lmbd = np.exp(0.5 * U_i * dt) + np.sqrt(np.expm1(U_i * dt))
    map_i = m["map_i"]
    d = {
        "metadata/commit": GEN_ID, "metadata/version": 0.1,
        "metadata/model": "Hubbard (complex)" if cplx else "Hubbard",
        "metadata/Nx": Nx, "metadata/Ny": Ny, "metadata/Norb": NORB[geometry],
        "metadata/bps": m["bps"], "metadata/b2ps": m["b2ps"],
        "metadata/plaq_per_cell": m["plaq_per_cell"], "metadata/U": U,
        "metadata/t'": tp, "metadata/t''": 0.0, "metadata/nflux": nflux, "metadata/twistx": 0,
        "metadata/twisty": 0, "metadata/mu": mu, "metadata/h": h, "metadata/beta": L * dt,
        "metadata/trans_sym": 1, "metadata/geometry": geometry, "metadata/bc": 1,
    }
    i32 = lambda v: np.array(v, dtype=np.int32)  # noqa: E731
    p = {
        "N": i32(N), "L": i32(L), "Nx": i32(Nx), "Ny": i32(Ny),
        "map_i": map_i, "map_ij": m["map_ij"], "bonds": m["bonds"], "plaqs": m["plaqs"],
        "map_plaq": m["map_plaq"], "map_b": m["map_b"], "map_bs": m["map_bs"],
        "map_bb": m["map_bb"], "peierlsu": ph, "peierlsd": ph.copy(),
        "Ku": Ku, "Kd": Kd, "U": U_i, "dt": np.array(dt, dtype=np.float64),
        "n_matmul": i32(n_matmul), "n_delay": i32(n_delay), "n_sweep_warm": i32(n_sweep_warm),
        "n_sweep_meas": i32(n_sweep_meas), "period_eqlt": i32(period_eqlt),
        "period_uneqlt": i32(period_uneqlt), "meas_bond_corr": meas_bond_corr,
        "meas_thermal": 0, "meas_2bond_corr": 0, "meas_energy_corr": 0, "meas_nematic_corr": 0,
        "meas_chiral": 0, "meas_local_JQ": 0, "meas_pair_bb_only": 0, "meas_gen_suscept": 0,
        "checkpoint_every": checkpoint_every,
        "num_i": i32(m["num_i"]), "num_ij": m["num_ij"], "num_plaq_accum": i32(m["num_plaq_accum"]),
        "num_b_accum": i32(m["num_b_accum"]), "num_b2_accum": i32(m["num_b2_accum"]),
        "num_plaq": m["num_plaq"], "num_b": m["num_b"], "num_b2": m["num_b2"],
        "num_bs": m["num_bs"], "num_bb": m["num_bb"], "num_b2b": m["num_b2b"],
        "num_bb2": m["num_bb2"], "num_b2b2": m["num_b2b2"],
        "degen_i": i32(m["degen_i"]), "degen_ij": i32(m["degen_ij"]),
        "degen_plaq": i32(m["degen_plaq"]), "degen_b": i32(m["degen_b"]),
        "degen_b2": i32(m["degen_b2"]), "degen_bs": i32(m["degen_bs"]),
        "degen_bb": i32(m["degen_bb"]), "degen_bb2": i32(m["degen_bb2"]),
        "degen_b2b": i32(m["degen_b2b"]), "degen_b2b2": i32(m["degen_b2b2"]),
        "exp_Ku": expm(-dt * Ku), "exp_Kd": expm(-dt * Kd),
        "inv_exp_Ku": expm(dt * Ku), "inv_exp_Kd": expm(dt * Kd),
        "exp_halfKu": expm(-dt / 2 * Ku), "exp_halfKd": expm(-dt / 2 * Kd),
        "inv_exp_halfKu": expm(dt / 2 * Ku), "inv_exp_halfKd": expm(dt / 2 * Kd),
        "exp_lambda": np.array((exp_lmbd[map_i] ** -1, exp_lmbd[map_i])),
        "del": np.array((exp_lmbd[map_i] ** 2 - 1, exp_lmbd[map_i] ** -2 - 1)),
        "F": i32(L // n_matmul), "n_sweep": i32(n_sweep_warm + n_sweep_meas),
    }
    for k, v in p.items():
        d["params/" + k] = v
    d.update(state_and_meas(N, L, init_rng, rng, hs, m, nt, period_uneqlt, meas_bond_corr))
    return d


def state_and_meas(N, L, init_rng, rng, hs, m, nt, period_uneqlt, meas_bond_corr) -> dict:
    """The state and zeroed measurement groups (gen_1band_unified_hub.py:1050-1160)."""
    nij, nbb = m["num_ij"], m["num_bb"]
    d = {"state/sweep": np.array(0, dtype=np.int32), "state/init_rng": init_rng,
         "state/rng": rng, "state/hs": hs, "state/partial_write": 0,
         "meas_eqlt/n_sample": np.array(0, dtype=np.int32),
         "meas_eqlt/sign": np.array(0.0, dtype=nt)}
    for k in ("density", "density_u", "density_d", "double_occ"):
        d["meas_eqlt/" + k] = np.zeros(m["num_i"], dtype=nt)
    for k in ("g00", "g00_u", "g00_d", "nn", "xx", "zz", "pair_sw"):
        d["meas_eqlt/" + k] = np.zeros(nij, dtype=nt)
    if period_uneqlt > 0:
        d["meas_uneqlt/n_sample"] = np.array(0, dtype=np.int32)
        d["meas_uneqlt/sign"] = np.array(0.0, dtype=nt)
        for k in ("gt0", "gt0_u", "gt0_d", "nn", "xx", "zz", "pair_sw"):
            d["meas_uneqlt/" + k] = np.zeros(nij * L, dtype=nt)
        if meas_bond_corr:
            for k in ("pair_bb", "jj", "jsjs", "kk", "ksks"):
                d["meas_uneqlt/" + k] = np.zeros(nbb * L, dtype=nt)
    return d


def chain_rngs(seed: int, n: int) -> list:
    """Per-chain initial RNG states as create_batch makes them: splitmix64 of
    the seed, then one 2^512 jump per further chain."""
    out = [seed_splitmix64(seed)]
    for _ in range(1, n):
        out.append(rand_jump(out[-1]))
    return out


def create_batch(Nfiles=1, prefix="sim", seed=0, **kw):
    """Write prefix_i.h5 for i < Nfiles plus prefix.h5.params, as the
    reference's create_batch (gen_1band_unified_hub.py:1163-1200)."""
    rngs = chain_rngs(seed, Nfiles)
    d0 = make_sim(init_rng=rngs[0], **kw)
    file_p = f"{prefix}.h5.params"
    params = {k: v for k, v in d0.items() if k.startswith(("metadata/", "params/"))}
    simfile.write(file_p, params)
    rel = os.path.basename(file_p)
    paths = []
    for i in range(Nfiles):
        if i == 0:
            d = d0
        else:
            N, L = int(d0["params/N"]), int(d0["params/L"])
            hs, rng = initial_hs(rngs[i], L, N)
            d = dict(d0)
            d["state/init_rng"], d["state/rng"], d["state/hs"] = rngs[i], rng, hs
        sim = {k: v for k, v in d.items() if not k.startswith(("metadata/", "params/"))}
        sim["params_file"] = rel
        sim["metadata"] = simfile.Link(rel)
        sim["params"] = simfile.Link(rel)
        path = f"{prefix}_{i}.h5"
        simfile.write(path, sim)
        paths.append(path)
    return paths


def make_ragged(n: int, seed: int, sides=(6, 8, 10, 14, 16), U=(2.0, 8.0), beta=(2.0, 8.0),
                dt: float = 0.05, n_matmul: int = 10, **kw) -> list:
    """Sim data of n chains with uneven lattices, U and beta: side uniform in
    `sides`, U and beta uniform in their ranges, L = beta / dt rounded to a
    multiple of n_matmul (the generator requires L % n_matmul == 0).  The
    per-chain draws come from numpy's PCG64 of `seed`; chain c's Markov
    chain starts from the master stream of `seed` jumped c times."""
    draw = np.random.Generator(np.random.PCG64(seed))
    rngs = chain_rngs(seed, n)
    period_eqlt = kw.pop("period_eqlt", n_matmul)
    out = []
    for c in range(n):
        side = int(draw.choice(np.asarray(sides)))
        u = float(draw.uniform(*U))
        b = float(draw.uniform(*beta))
        L = max(n_matmul, int(round(b / dt / n_matmul)) * n_matmul)
        out.append(make_sim(Nx=side, Ny=side, U=u, dt=dt, L=L, n_matmul=n_matmul,
                            init_rng=rngs[c], period_eqlt=period_eqlt, **kw))
    return out
