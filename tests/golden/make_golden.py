"""Regenerate the golden fixtures under tests/golden/.

Runs where the reference checkout is present only (it reads it at
$DQMC_REF_ROOT, default: a "reference" folder beside this repository):

* sim inputs come from the reference generator util/gen_1band_unified_hub.py
  (create_batch), run with the h5py/git stand-ins in _stubs/ so that it writes
  DQSF containers;
* reference outputs come from the reference's own C (src/*.c) built by
  `make -C oracle ref` into oracle/_ref/dqmc_1_{r,c}, run on a copy of each
  input;
* hs_ref.npz holds the reference test suite's golden HS fields
  (test/hs_ref.py), for the 4-geometry known-answer test.

Usage:  python tests/golden/make_golden.py [case ...]
"""
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_ROOT = os.environ.get("DQMC_REF_ROOT", os.path.join(ROOT, "..", "reference"))
sys.path.insert(0, os.path.join(HERE, "_stubs"))
sys.path.insert(0, os.path.join(REF_ROOT, "util"))
sys.path.insert(0, os.path.join(REF_ROOT, "test"))
sys.path.insert(0, os.path.join(ROOT, "dqmc-dev_b200"))

import gen_1band_unified_hub as ghub  # noqa: E402
import gen_util_shared as gus  # noqa: E402
import hs_ref  # noqa: E402
from dqmc_b200 import simfile  # noqa: E402

GEOMETRIES = ["square", "triangular", "honeycomb", "kagome"]

CASES = {
    # test_batch_seed_basic_real (test/test_gen_1band_hub_unified.py:119-148)
    **{f"kat_{g}": dict(geometry=g, seed=1234, n_sweep_warm=20, n_sweep_meas=20)
       for g in GEOMETRIES},
    # the small single-chain configuration: 4x4, U=4, beta=4, n_matmul=5, delay 8
    "c1_small": dict(geometry="square", seed=7, Nx=4, Ny=4, U=4.0, mu=0.0, dt=0.1,
                     L=40, n_matmul=5, n_delay=8, period_eqlt=8,
                     n_sweep_warm=10, n_sweep_meas=20),
    # unequal-time + bond correlators, t' and mu != 0
    "uneq_small": dict(geometry="square", seed=11, Nx=4, Ny=4, tp=-0.25, U=6.0,
                       mu=-0.5, dt=0.1, L=16, n_matmul=4, n_delay=4, period_eqlt=4,
                       period_uneqlt=2, meas_bond_corr=1, n_sweep_warm=4,
                       n_sweep_meas=8),
    # odd F (uneven cluster grouping in calc_eq_g and bsofi)
    "uneq_oddF": dict(geometry="square", seed=5, Nx=4, Ny=4, U=4.0, mu=-0.3, dt=0.1,
                      L=30, n_matmul=6, n_delay=5, period_eqlt=5, period_uneqlt=1,
                      meas_bond_corr=1, n_sweep_warm=2, n_sweep_meas=4),
    # complex hoppings: Peierls flux through the 4x4 torus
    "cplx_small": dict(geometry="square", seed=3, Nx=4, Ny=4, nflux=1, U=4.0, mu=0.0,
                       dt=0.1, L=20, n_matmul=5, n_delay=4, period_eqlt=5,
                       period_uneqlt=2, meas_bond_corr=1, n_sweep_warm=2,
                       n_sweep_meas=6),
    # every measurement toggle (t' != 0 gives the square lattice's full
    # bond and two-bond families)
    "tog_sq": dict(geometry="square", seed=41, Nx=4, Ny=4, tp=-0.25, U=4.0, mu=-0.3,
                   dt=0.1, L=16, n_matmul=4, n_delay=4, period_eqlt=4, period_uneqlt=2,
                   meas_bond_corr=1, meas_energy_corr=1, meas_thermal=1, meas_2bond_corr=1,
                   meas_nematic_corr=1, meas_chiral=1, meas_gen_suscept=1,
                   n_sweep_warm=2, n_sweep_meas=4),
    # the toggles with Peierls phases (the reference has no complex nematic)
    "tog_cplx": dict(geometry="square", seed=42, Nx=4, Ny=4, nflux=1, tp=-0.25, U=4.0,
                     mu=-0.3, dt=0.1, L=16, n_matmul=4, n_delay=4, period_eqlt=4,
                     period_uneqlt=2, meas_bond_corr=1, meas_energy_corr=1, meas_thermal=1,
                     meas_2bond_corr=1, meas_chiral=1, meas_gen_suscept=1,
                     n_sweep_warm=2, n_sweep_meas=4),
    # the toggles that need trans_sym = 0: local heat current, pair_bb only
    "tog_local": dict(geometry="square", seed=43, Nx=4, Ny=4, tp=-0.25, U=4.0, mu=-0.3,
                      dt=0.1, L=16, n_matmul=4, n_delay=4, period_eqlt=4, period_uneqlt=2,
                      trans_sym=0, meas_local_JQ=1, meas_pair_bb_only=1,
                      n_sweep_warm=2, n_sweep_meas=4),
    # a larger lattice, for kernels that tile N (N = 64)
    "sq8_small": dict(geometry="square", seed=21, Nx=8, Ny=8, tp=-0.25, U=6.0,
                      mu=-0.5, dt=0.1, L=16, n_matmul=8, n_delay=16, period_eqlt=8,
                      n_sweep_warm=2, n_sweep_meas=2),
}

# generator-only cases: parameters are compared with the engine's own generator
GEN_CASES = {
    "gen_sq6_tp": dict(geometry="square", seed=1, Nx=6, Ny=6, tp=-0.25, U=6.0, mu=-0.5,
                       dt=0.1, L=20, n_matmul=5, n_delay=8, period_eqlt=5,
                       period_uneqlt=1, meas_bond_corr=1),
    "gen_sq4_flux": dict(geometry="square", seed=2, Nx=4, Ny=4, nflux=1, U=4.0, mu=0.0,
                         dt=0.1, L=20, n_matmul=5, n_delay=8, period_eqlt=5),
    "gen_sq6_flux": dict(geometry="square", seed=4, Nx=6, Ny=6, nflux=1, U=4.0,
                         dt=0.1, L=10, n_matmul=5, n_delay=8, period_eqlt=5),
    "gen_sq4_h": dict(geometry="square", seed=9, Nx=4, Ny=6, U=3.0, mu=0.2, h=0.1,
                      dt=0.05, L=20, n_matmul=10, n_delay=8, period_eqlt=10),
    # Peierls phases with sublattice offsets on the other lattices
    "gen_tri_flux": dict(geometry="triangular", seed=31, Nx=4, Ny=4, nflux=1, U=4.0,
                         mu=-0.2, dt=0.1, L=10, n_matmul=5, n_delay=8, period_eqlt=5),
    "gen_hc_flux": dict(geometry="honeycomb", seed=32, Nx=3, Ny=3, nflux=1, U=4.0,
                        dt=0.1, L=10, n_matmul=5, n_delay=8, period_eqlt=5),
    "gen_kag_flux": dict(geometry="kagome", seed=33, Nx=3, Ny=3, nflux=2, U=4.0,
                         mu=0.3, dt=0.1, L=10, n_matmul=5, n_delay=8, period_eqlt=5),
}


def generate(case_dir, kw):
    os.makedirs(case_dir, exist_ok=True)
    cwd = os.getcwd()
    os.chdir(case_dir)
    try:
        for f in os.listdir("."):
            if f.endswith(".h5") or f.endswith(".params"):
                os.remove(f)
        ghub.create_batch(overwrite=1, **kw)
    finally:
        os.chdir(cwd)


# datasets no engine path reads (two-bond maps and phases, plaquettes); they
# are dropped from the committed copies to keep the fixtures small
DROP = ("bond2s", "map_b2", "map_b2b", "map_bb2", "map_b2b2", "pp_u", "pp_d",
        "ppr_u", "ppr_d", "map_bs", "plaqs", "map_plaq")


TOGGLES = ("meas_thermal", "meas_2bond_corr", "meas_energy_corr", "meas_nematic_corr",
           "meas_chiral", "meas_local_JQ", "meas_gen_suscept", "meas_pair_bb_only")


def compact(case_dir):
    """drop the maps no engine path reads, unless a measurement toggle that
    reads them is on"""
    path = os.path.join(case_dir, "sim.h5.params")
    d = simfile.read(path, resolve_links=False)
    if any(int(np.asarray(d.get("params/" + t, 0)).reshape(-1)[0]) for t in TOGGLES):
        return
    keep = {k: v for k, v in d.items() if k.split("/")[-1] not in DROP}
    simfile.write(path, keep)


def run_reference(case_dir, cplx):
    exe = os.path.join(ROOT, "oracle", "_ref", "dqmc_1_c" if cplx else "dqmc_1_r")
    with tempfile.TemporaryDirectory() as tmp:
        for f in ("sim_0.h5", "sim.h5.params"):
            shutil.copy(os.path.join(case_dir, f), tmp)
        env = dict(os.environ, OPENBLAS_NUM_THREADS="1")
        subprocess.run([exe, "-l", os.path.join(tmp, "log"), os.path.join(tmp, "sim_0.h5")],
                       check=True, env=env)
        d = simfile.read(os.path.join(tmp, "sim_0.h5"))
    out = {k.replace("/", "__"): np.asarray(v) for k, v in d.items()
           if k.startswith(("state/", "meas_eqlt/", "meas_uneqlt/"))}
    np.savez(os.path.join(case_dir, "ref_out.npz"), **out)


def main(only=()):
    """all fixtures, or only the named cases"""
    if only:
        for name in only:
            if name in GEN_CASES:
                generate(os.path.join(HERE, name), GEN_CASES[name])
                compact(os.path.join(HERE, name))
            else:
                kw = CASES[name]
                generate(os.path.join(HERE, name), kw)
                run_reference(os.path.join(HERE, name), cplx=kw.get("nflux", 0) != 0)
                compact(os.path.join(HERE, name))
            print("case", name, "done")
        return
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    np.savez(os.path.join(HERE, "hs_ref.npz"),
             **{f"init_{g}": hs_ref.hs_init[g] for g in GEOMETRIES},
             **{f"end_{g}": hs_ref.hs_end[g] for g in GEOMETRIES})
    # RNG vectors from the reference generator's helpers (gen_util_shared.py)
    seeded = gus.rand_seed_splitmix64(1234)
    jumped = seeded.copy()
    gus.rand_jump(jumped)
    draws = seeded.copy()
    first = np.array([gus.rand_uint(draws) for _ in range(64)], dtype=np.uint64)
    np.savez(os.path.join(HERE, "rng_ref.npz"), seed=np.uint64(1234), seeded=seeded,
             jumped=jumped, first_draws=first, state_after=draws)
    for name, kw in CASES.items():
        d = os.path.join(HERE, name)
        generate(d, kw)
        run_reference(d, cplx=kw.get("nflux", 0) != 0)
        compact(d)
        print("case", name, "done")
    for name, kw in GEN_CASES.items():
        generate(os.path.join(HERE, name), kw)
        compact(os.path.join(HERE, name))
        print("generator case", name, "done")


if __name__ == "__main__":
    main(sys.argv[1:])
