"""Writes tests/golden/*.npz: small cases of the GDF P2 step computed by the
CPU oracle (oracle/gdf_oracle.cpp, the restatement of the reference), used
as committed fixtures by tests/test_golden.py. The reference ships no
golden vectors and its Fortran cannot be built here, so these pin the
oracle against its own past outputs (regressions) and let the GPU tests
check the library without building the oracle.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "freljord-cfd-arsenal_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

import gdf  # noqa: E402
from oracle import Oracle  # noqa: E402

# name: (problem, nx, ny, config edits, steps)
CASES = {
    "ot_hll_all_10x8": (gdf.PROB_ORSZAG_TANG, 10, 8, {}, 3),
    "rotor_hlld_kxrcf_pp_12x12": (gdf.PROB_ROTOR, 12, 12, {"faceb_limiter": 0}, 3),   # raw face B
    "blast_hlld_faceb_10x12": (gdf.PROB_BLAST, 10, 12, {}, 3),
    "cloud_hllc_12x6": (gdf.PROB_CLOUD_SHOCK, 12, 6, {"flux_type": gdf.FLUX_HLLC}, 2),
    "vortex_lf_8x8": (gdf.PROB_VORTEX, 8, 8, {"flux_type": gdf.FLUX_LF}, 2),
    "rotor_df_variant_12x10": (gdf.PROB_ROTOR, 12, 10,
                               {"cfl": 0.2, "hlld_eps": 1e-12, "tvb_slope": 2.0 / 3.0, "faceb_limiter": 1,
                                "ez_face_fhat": 1, "eig_p_typo": 1, "eig_identity": 0, "eig_y_zero_w": 1,
                                "kml_w_term": 0, "dt_floor_stop": 0, "umax_all_vars": 1}, 2),
}


def case_config(name):
    prob, nx, ny, edits, steps = CASES[name]
    cfg, _ = gdf.problem_config(prob, nx, ny)
    for k, v in edits.items():
        setattr(cfg, k, v)
    return cfg, prob, steps


def run_oracle(name):
    cfg, prob, steps = case_config(name)
    o = Oracle(cfg)
    uh, bx, by = o.init_data(prob)
    init = (uh.copy(), bx.copy(), by.copy())
    fp = o.prepare(uh, bx, by)
    flags = [fp]
    ts, dts = [], []
    t = 0.0
    for _ in range(steps):
        t, dt, f = o.step(uh, bx, by, t, 1e9)
        flags.append(f)
        ts.append(t)
        dts.append(dt)
    return {"uh0": init[0], "bx0": init[1], "by0": init[2], "uh": uh, "bx": bx, "by": by,
            "flags": np.stack(flags), "t": np.array(ts), "dt": np.array(dts)}


def main():
    for name in CASES:
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **run_oracle(name))
        print("wrote", name)


if __name__ == "__main__":
    main()
