"""Generate the golden fixtures in tests/golden/ from the reference itself.

The reference (its own C sources, compiled unmodified against this project's
single-rank MPI/FFTW-API shims into oracle/_ref/libmhdref.so by
oracle/Makefile) is run on small seeded inputs; its outputs are saved as
compressed .npz files.  Run from the repository root:

    make -C oracle && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import ref  # noqa: E402
from mhd2dcfdfftw_open_b200 import ic  # noqa: E402


def rand_state(p, seed):
    rng = np.random.default_rng(seed)
    uu = rng.standard_normal(p.state_shape())
    uu[0] = 1.5 + 0.3 * np.abs(uu[0])
    uu[7] = 1.0 + 0.3 * np.abs(uu[7])
    return uu


def params_dict(p):
    return {k: np.array(v) for k, v in vars(p).items()}


def main():
    R = ref.Reference()
    # per-operator fixtures on random fields
    for nx, ny, seed in ((16, 16, 11), (40, 8, 12), (24, 32, 13)):
        p, _ = ic.orszag_tang(nx, ny, di=0.05)
        R.setup(p)
        uu = rand_state(p, seed)
        out = dict(uu=uu,
                   derivX=R.deriv_x(uu, 1), derivXX=R.deriv_x(uu, 2),
                   derivY=R.deriv_y(uu, 1), derivYY=R.deriv_y(uu, 2),
                   filtering=R.filtering(uu))
        R.setup(p)
        dt, _, _ = R.calc_dt(uu, 0.0)
        out["calcDt"] = np.array(dt)
        np.savez_compressed(os.path.join(HERE, f"ops_{nx}x{ny}.npz"), **out,
                            **{"p_" + k: v for k, v in params_dict(p).items()})
    # whole steps
    cases = [
        ("ot_32x32_di005", ic.orszag_tang(32, 32, di=0.05), 1e-3, (1, 10)),
        ("ot_32x32_di0", ic.orszag_tang(32, 32, di=0.0), 1e-3, (1,)),
        ("ot_32x16_clean1", ic.orszag_tang(32, 16, di=0.05, divBcleaning=1), 1e-3, (2,)),
        ("ot_32x16_clean2", ic.orszag_tang(32, 16, di=0.05, divBcleaning=2), 1e-3, (2,)),
        ("ot_32x16_cfl", ic.orszag_tang(32, 16, di=0.05), -1.0, (3,)),
        ("turb_32x32", ic.alfvenic_turbulence(32, 32, mmax=6), 2e-4, (1,)),
    ]
    for name, (p, uu), dt_fixed, nsteps_list in cases:
        if p.divBcleaning == 2:
            rng = np.random.default_rng(7)
            uu[8] = 1e-3 * rng.standard_normal(uu.shape[1:])
        out = {"uu0": uu}
        for n in nsteps_list:
            R.setup(p)
            R.set_state(uu)
            _, dt = R.steps(n, dt_fixed)
            out[f"uu_{n}"] = R.uu.copy()
            out[f"dt_{n}"] = np.array(dt)
            out[f"maxdivb_{n}"] = np.array(R.check_divb())
        out["dt_fixed"] = np.array(dt_fixed)
        np.savez_compressed(os.path.join(HERE, f"steps_{name}.npz"), **out,
                            **{"p_" + k: v for k, v in params_dict(p).items()})
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
