"""Writes the golden fixtures the parity tests read.

Run where the edge-rs 0.4.0 sources are checked out (read-only), naming
their root on the command line or in EDGE_RS_REFERENCE:

    python tests/golden/make_goldens.py <edge-rs root>

1. Copies the reference's committed R-derived CSV fixtures (produced by its
   tests/r/generate_fixtures.R from nebula 1.5.8/1.5.9 and nloptr 2.2.1) into
   tests/golden/data/: the BOBYQA traces, the 8-gene x 150-cell NEBULA golden
   and the end-to-end datasets (NEBULA-HL and NEBULA-LN).
2. Writes tests/golden/inline_goldens.json: the literal expected values the
   reference keeps inside its unit tests (R's 17-digit prints), transcribed
   here with the file:line each comes from.

The tests read only the files this script writes, so they run where no copy
of the reference exists.
"""
import json
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "data")

# NEBULA-HL datasets of tests/e2e_nebula.rs:288-398 (method HL, or LN below 30
# cells per subject, which the driver turns into HL), plus the LN ones kept for
# the LN path.
E2E_HL = ["sc_small", "sc_k2", "sc_intercept", "sc_wide", "sc_high", "sc_cat_hl", "sc_cat_sparse"]
E2E_LN = ["sc_blocks", "sc_cat_ln", "sc", "sc_xwide"]
BOBYQA = ["rosen", "rosen_edge", "corner", "chain3", "rescue", "roundoff"]

# --- opt_pml goldens, src/sc/pml.rs:2149-2700 (nebula:::opt_pml, nebula 1.5.8) ---
PML_FIXTURE_A = {
    "design": [1.0, 0.0, 1.0, 1.0, 1.0, 0.0, 1.0, 1.0, 1.0, 1.0, 1.0, 0.0, 1.0, 1.0, 1.0, 0.0,
               1.0, 1.0, 1.0, 0.0, 1.0, 1.0, 1.0, 1.0],  # pml.rs:2151-2154
    "offset": [0.25, -0.5, 0.75, 0.0, 0.5, -0.25, 0.125, 0.375, -0.125, 0.25, 0.0, -0.375],
    "subject_start": [0, 4, 9, 12],
    "counts": [3.0, 5.0, 2.0, 4.0, 1.0, 7.0, 2.0, 6.0],
    "cells": [0, 2, 3, 5, 6, 7, 9, 10],
    "subject_total": [10.0, 12.0, 8.0],
}
PML_FIXTURE_B = dict(PML_FIXTURE_A, counts=[3.0, 5.0, 2.0, 2.0, 6.0], cells=[0, 2, 3, 9, 10],
                     subject_total=[10.0, 0.0, 8.0])  # pml.rs:2173-2180

PML_CASES = [
    {"name": "well_behaved", "src": "src/sc/pml.rs:2232-2265", "fixture": "A",
     "beta_init": [0.5, -0.25], "subject": 0.25, "cell": 2.0,
     "beta": [1.1055943907637618, -0.98348970166026206],
     "log_w": [-0.025429869309964156, 0.022419629678247836, 0.33781545877640862],
     "information": [5.4708370512237092, 2.6193993778249318, 2.6193993778249318, 4.0223986651682804],
     "log_likelihood": -60.378642466146786, "log_det": 6.0421923783970968,
     "second_order": 0.0, "iterations": 4, "backtracks": 0, "convergence": 1},
    {"name": "third_order", "src": "src/sc/pml.rs:2267-2283", "fixture": "A", "ord": 3,
     "beta_init": [0.5, -0.25], "subject": 0.25, "cell": 2.0,
     "beta": [1.1055943907637618, -0.98348970166026206], "second_order": 0.0028301625845031939},
    {"name": "reml", "src": "src/sc/pml.rs:2285-2300", "fixture": "A", "reml": True,
     "beta_init": [0.5, -0.25], "subject": 0.25, "cell": 2.0,
     "log_det": 8.759838692617901, "beta": [1.1055943907637618, -0.98348970166026206]},
    {"name": "all_zero_subject", "src": "src/sc/pml.rs:2302-2332", "fixture": "B",
     "beta_init": [0.5, -0.25], "subject": 0.25, "cell": 2.0,
     "beta": [0.15781792039265752, -0.098178037869394941],
     "log_w": [0.31781101972092152, -0.83477809302857631, 0.46458776408134972],
     "information": [4.9151627959404793, 2.59325292186585, 2.59325292186585, 3.5781777249175555],
     "log_likelihood": -50.769290856943599, "log_det": 5.3802869340559738, "convergence": 1},
    {"name": "zero_subject_third_order", "src": "src/sc/pml.rs:2334-2347", "fixture": "B",
     "ord": 3, "beta_init": [0.5, -0.25], "subject": 0.25, "cell": 2.0,
     "second_order": 0.029026901671004347},
    {"name": "start_near_bound", "src": "src/sc/pml.rs:2349-2380", "fixture": "A",
     "beta_init": [90.0, 0.0], "subject": 0.25, "cell": 2.0,
     "beta": [1.1055943759446161, -0.98348968952057669],
     "log_w": [-0.025429869876909816, 0.022419639320108459, 0.3378154594265026],
     "information": [5.4711020927179739, 2.6193969725187061, 2.6193969725187061, 4.0224446400576319],
     "iterations": 9, "convergence": 1},
    {"name": "fixed_displacement", "src": "src/sc/pml.rs:2382-2396", "fixture": "A",
     "beta_init": [-90.0, 60.0], "subject": 0.25, "cell": 2.0,
     "beta": [1.1055943725487707, -0.98348968650982715], "log_det": 6.0423215051590002,
     "iterations": 12},
    {"name": "critical_point", "src": "src/sc/pml.rs:2398-2425", "fixture": "A",
     "beta_init": [15.0, 5.0], "subject": 8.0, "cell": 0.001,
     "beta": [4.9609375, -4.9609375], "log_w": [0.0390625, 0.0390625, 4.5234136840078936],
     "information": [7.0733722800021132e-05, 7.0105348391562988e-05, 7.0105348391562988e-05,
                     0.00016310178559274507],
     "log_det": -20.515549220945573, "iterations": 3, "backtracks": 11, "convergence": -10},
    {"name": "stalled", "src": "src/sc/pml.rs:2427-2441", "fixture": "A",
     "beta_init": [20.0, 0.0], "subject": 8.0, "cell": 0.001,
     "beta": [14.9609375, -4.9609375], "log_w": [-4.9609375, -4.9609375, 4.9962571608576489],
     "iterations": 2, "backtracks": 12, "convergence": -40},
    {"name": "iteration_budget", "src": "src/sc/pml.rs:2443-2469", "fixture": "A", "eps": -1e-300,
     "beta_init": [0.5, -0.25], "subject": 0.25, "cell": 2.0, "iterations": 50, "convergence": -20,
     "beta": [1.1055943907637629, -0.98348970166026151],
     "information": [5.4708368635191373, 2.619399280826618, 2.619399280826618, 4.0223986123865263]},
    {"name": "collinear", "src": "src/sc/pml.rs:2471-2500", "fixture": "A", "design": "collinear",
     "beta_init": [0.5, -0.25, 0.1], "subject": 0.25, "cell": 2.0, "convergence": -25,
     "beta": [1.1055943330380458, -1.0834897078722583, 0.10000000000000001],
     "log_det": 6.042689573294485},
    {"name": "single_coefficient", "src": "src/sc/pml.rs:2502-2536", "fixture": "A",
     "design": "ones", "reml": True, "ord": 3, "beta_init": [0.0], "subject": 0.25, "cell": 2.0,
     "beta": [0.64526354365336647],
     "log_w": [0.040002950937536336, 0.10805651074009694, 0.21875064209166895],
     "information": [5.7533150000267472], "log_det": 7.9235375511695514,
     "second_order": 0.0044134970888637676},
    {"name": "nbm", "src": "src/sc/pml.rs:2538-2574", "fixture": "A", "prior": "lognormal",
     "reml": True, "beta_init": [0.5, -0.25], "subject": 0.3, "cell": 2.0,
     "beta": [1.2213403122060453, -0.98985988766009869],
     "log_w": [-0.14301073703498665, -0.095894342874540239, 0.23890507990952689],
     "information": [5.4025646031315233, 2.5076353884976541, 2.5076353884976541, 3.9141513741254204],
     "log_likelihood": -49.318101708775217, "log_det": 8.6579114426780528, "second_order": 0.0,
     "iterations": 3, "convergence": 1},
    {"name": "wider_design", "src": "src/sc/pml.rs:2634-2700", "fixture": "large", "reml": True,
     "ord": 3, "beta_init": [0.5, -0.25, 0.75], "subject": 0.35, "cell": 1.5,
     "beta": [1.4272053191863423, 0.20743588590645803, -0.017982095723719935],
     "log_w": [0.21944093016930771, 0.12415265795703513, 0.20913336580790309, 0.14393280971073011],
     "information": [8.398261243665857, 2.7062153540842324, 3.0637064599168475, 2.7062153540842324,
                     16.226178650135836, 1.2821611476475319, 3.0637064599168475, 1.2821611476475319,
                     5.5864643706193053],
     "log_likelihood": -276.5244116459354, "log_det": 18.407453390744379,
     "second_order": 0.0029993806316514779, "iterations": 4, "convergence": 1},
    {"name": "wider_design_plain", "src": "src/sc/pml.rs:2695-2699", "fixture": "large",
     "beta_init": [0.5, -0.25, 0.75], "subject": 0.35, "cell": 1.5,
     "beta": [1.4272053191863423, 0.20743588590645803, -0.017982095723719935],
     "log_det": 12.052188343414912, "second_order": 0.0},
]

# pml_ll_der_eigen at a point, src/sc/pml.rs:2576-2600
PML_GRADIENT = {"src": "src/sc/pml.rs:2576-2600", "beta": [0.5, -0.25],
                "log_w": [0.1, -0.2, 0.05], "subject": 0.25, "cell": 2.0,
                "objective": 53.926203132942852,
                "gradient": [-5.2597994101747254, -0.19846989257393055, -0.40624529144311583,
                             -2.8367693486273806, -2.0229915782218155]}

# --- stage-one marginal likelihood goldens, src/sc/ptmg.rs:2018-2442 ---
PTMG_FIXTURES = {
    "A": {"x": [[0.0], [1.0], [0.5], [-0.5], [0.25], [-1.0]],  # ptmg.rs:2026-2043
          "log_offset": [0.0, 0.25, -0.5, 0.125, 0.75, -0.25],
          "counts": [3.0, 1.0, 2.0, 5.0], "cells": [0, 2, 3, 5],
          "subject_totals": [3.0, 3.0, 5.0], "fid": [0, 2, 5, 6]},
    "B": {"x": [[0.0, 0.5], [1.0, -0.25], [0.5, 0.0], [-0.5, 0.75], [0.25, -1.0], [-1.0, 0.25],
                [0.75, 1.0], [-0.25, -0.5]],  # ptmg.rs:2052-2074
          "log_offset": [0.5, -0.25, 0.125, 0.0, 0.375, -0.75, 0.25, 1.0],
          "counts": [2.0, 1.0, 4.0, 1.0, 7.0], "cells": [1, 2, 4, 6, 7],
          "subject_totals": [3.0, 0.0, 12.0], "fid": [0, 3, 4, 8]},
}
PTMG_CASES = [
    {"src": "src/sc/ptmg.rs:2162-2195", "fixture": "A", "params": [0.5, -0.25, 0.5, 2.0],
     "value": 5.68919227265053351e+00, "gtol": 1e-10, "htol": 1e-8,
     "gradient": [1.23230096727342087e-01, 2.14374578345666933e+00, 1.96862959139235372e+00,
                  -1.46930062054576371e-01],
     "hessian": [2.46157581206725151e+00, -7.12808069390344246e-01, 2.39173560205083291e-01,
                 -2.69050975196676243e-02, -7.12808069390344246e-01, 2.05333290435219373e+00,
                 -1.34438513739700594e+00, 3.31302601132097918e-01, 2.39173560205083291e-01,
                 -1.34438513739700594e+00, 3.91220510021810242e-02, -1.42705917336173937e-01,
                 -2.69050975196676243e-02, 3.31302601132097918e-01, -1.42705917336173937e-01,
                 1.68849516491021756e-01]},
    {"src": "src/sc/ptmg.rs:2197-2232", "fixture": "A", "params": [1.25, 0.75, 1e-4, 1e-4],
     "value": 3.29896692291768900e+01, "gtol": 1e-8, "htol": 1e-6,
     "gradient": [2.96406695818021149e-02, 1.31693015791212176e-02, 1.30305458759699832e+02,
                  -3.99414489355896367e+04],
     "hessian": [6.86679893234001110e-02, 2.79446317794878468e-02, 2.95430767492699658e+02,
                 1.82090109226938218e-01, 2.79446317794878468e-02, 2.14302885561563627e-02,
                 1.27035501836412706e+02, 4.34573972169806044e+00, 2.95430767492699658e+02,
                 1.27035501836412706e+02, -4.52776105356216431e+03, -4.46684522479116310e+01,
                 1.82090109226938218e-01, 4.34573972169806044e+00, -4.46684522479116310e+01,
                 3.99940003972201765e+08]},
    {"src": "src/sc/ptmg.rs:2234-2268", "fixture": "A", "params": [-0.5, 0.125, 8.0, 512.0],
     "value": 2.65308778580696725e+01, "gtol": 1e-10, "htol": 1e-8,
     "gradient": [9.12793250876120510e-04, 2.53045547739533250e+00, 2.99186987816233607e+00,
                  -3.60045252223439860e-07],
     "hessian": [9.39311823971149956e-05, -6.57328696371346430e-05, -8.66127875657092474e-04,
                 3.13400144628472963e-11, -6.57328696371346430e-05, 1.13575813292771000e+00,
                 9.98036672113045331e-06, 1.32876795203876600e-05, -8.66127875657092474e-04,
                 9.98036672113045331e-06, 6.69606190840976723e-03, -1.05310011543468632e-09,
                 3.13400144628472963e-11, 1.32876795203876600e-05, -1.05310011543468632e-09,
                 1.36270078923174387e-09]},
    {"src": "src/sc/ptmg.rs:2270-2304", "fixture": "A", "params": [0.0, 0.0, 2.0, 0.25],
     "value": 1.12063514415980094e+01, "gtol": 1e-10, "htol": 1e-8,
     "gradient": [-3.81456775084743072e-03, 5.74173792151410289e-01, 2.38393039589584355e+00,
                  -7.26967190944776576e+00],
     "hessian": [4.23398202512259736e-01, -2.57145238578597779e-01, 1.94645018901316025e-01,
                 -1.15565351220650037e-02, -2.57145238578597779e-01, 7.01861921458433624e-01,
                 -3.59445802666915337e-01, 1.18270172064454471e+00, 1.94645018901316025e-01,
                 -3.59445802666915337e-01, 4.36597493935281022e-01, 1.30165671415671189e-02,
                 -1.15565351220650037e-02, 1.18270172064454471e+00, 1.30165671415671189e-02,
                 4.50117573398768016e+01]},
    {"src": "src/sc/ptmg.rs:2306-2350", "fixture": "B", "params": [0.25, -0.5, 0.75, 1.5, 3.0],
     "value": 7.46199076417621399e+00, "gtol": 1e-10, "htol": 1e-8,
     "gradient": [5.01350696391867245e-01, -2.04257563318932167e+00, 5.34153324797603979e+00,
                  1.07011331098338225e+00, 2.53578958023772838e-01],
     "hessian": [3.48740746684502056e-01, 2.54876819316399161e-02, 1.45533761085350766e-02,
                 -4.41548536268330516e-01, 3.91566084164468586e-03, 2.54876819316399161e-02,
                 2.09570270083503551e+00, 2.64460193688231204e-01, 1.02670366878276728e-01,
                 -5.76636821621331688e-02, 1.45533761085350766e-02, 2.64460193688231204e-01,
                 3.84459569945194923e+00, -2.78923375808989293e-01, 6.39405403297957253e-01,
                 -4.41548536268330516e-01, 1.02670366878276728e-01, -2.78923375808989293e-01,
                 3.66772893546357448e-01, -1.49218225719068356e-02, 3.91566084164468586e-03,
                 -5.76636821621331688e-02, 6.39405403297957253e-01, -1.49218225719068356e-02,
                 -7.22442940506229370e-02]},
    {"src": "src/sc/ptmg.rs:2352-2396", "fixture": "B", "params": [-1.0, 0.5, 0.25, 1e-4, 1000.0],
     "value": 1.13584681060607693e+01, "gtol": 1e-8, "htol": 1e-6,
     "gradient": [-1.07326878153205776e+01, -1.48756816066168707e+00, 7.53628836395186852e+00,
                  -4.62797267317655496e+01, 1.95947859886434761e-05],
     "hessian": [4.26381285975427904e+00, 1.01145653996075602e+00, 5.35701406304531225e-01,
                 2.61662160722283907e+01, -6.94406121181113076e-06, 1.01145653996075602e+00,
                 1.35186752241846908e+00, 3.72773749626097717e-01, 6.11253074542543828e+00,
                 -1.69452414787726765e-07, 5.35701406304531225e-01, 3.72773749626097717e-01,
                 1.95363290656862110e+00, 9.21736461732613921e-01, 4.48552067926583857e-06,
                 2.61662160722283907e+01, 6.11253074542543828e+00, 9.21736461732613921e-01,
                 4.35795623779296875e+02, -6.84104019316582210e-05, -6.94406121181113076e-06,
                 -1.69452414787726765e-07, 4.48552067926583857e-06, -6.84104019316582210e-05,
                 -3.90898716648611179e-08]},
    {"src": "src/sc/ptmg.rs:2398-2442", "fixture": "B", "params": [0.75, -0.25, 0.5, 10.0, 1e-4],
     "value": 5.76091855400661359e+01, "gtol": 1e-10, "htol": 1e-8,
     "gradient": [1.35773392448967911e-04, -3.59794963305848370e-04, 4.96443874810736929e-04,
                  1.99820940875096320e+00, -4.99346186500725235e+04],
     "hessian": [4.32580556442951729e-07, 4.91633557431160259e-08, 2.83994566060920446e-08,
                 -1.35563254538641632e-04, -9.85888077842389521e-08, 4.91633557431160259e-08,
                 3.29393259974663849e-04, -2.02106061975382121e-04, 7.65773286491442306e-06,
                 -3.52089986509287156e+00, 2.83994566060920446e-08, -2.02106061975382121e-04,
                 4.54276735397987554e-04, -4.52632990189595600e-05, 4.51109987283559022e+00,
                 -1.35563254538641632e-04, 7.65773286491442306e-06, -4.52632990189595600e-05,
                 1.57701505319085555e-03, -9.74640513908427847e-02, -9.85888077842389521e-08,
                 -3.52089986509287156e+00, 4.51109987283559022e+00, -9.74640513908427847e-02,
                 4.99929026939662099e+08]},
]


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("EDGE_RS_REFERENCE")
    if not ref or not os.path.isdir(os.path.join(ref, "tests", "data")):
        sys.exit("usage: make_goldens.py <edge-rs root> (or set EDGE_RS_REFERENCE)")
    os.makedirs(DATA, exist_ok=True)
    files = [f"e2e/bobyqa_{t}.csv" for t in BOBYQA]
    for tag in E2E_HL + E2E_LN:
        for part in ("counts", "meta", "design", "nebula", "covariance"):
            p = f"e2e/{tag}_{part}.csv"
            if os.path.exists(os.path.join(ref, "tests", "data", p)):
                files.append(p)
    files += ["e2e/scalars.csv"]
    files += [f"nebula_{p}.csv" for p in ("counts", "design", "expected", "covariance")]
    for f in files:
        shutil.copyfile(os.path.join(ref, "tests", "data", f), os.path.join(DATA, os.path.basename(f)))
    inline = {"pml_fixture_a": PML_FIXTURE_A, "pml_fixture_b": PML_FIXTURE_B, "pml_cases": PML_CASES,
              "pml_gradient": PML_GRADIENT, "ptmg_fixtures": PTMG_FIXTURES, "ptmg_cases": PTMG_CASES,
              "e2e_hl": E2E_HL, "e2e_ln": E2E_LN, "bobyqa": BOBYQA}
    with open(os.path.join(HERE, "inline_goldens.json"), "w") as fh:
        json.dump(inline, fh, indent=1)
    print(f"copied {len(files)} fixtures into {DATA}")


if __name__ == "__main__":
    main()
