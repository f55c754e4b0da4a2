"""Generates the golden fixtures in tests/golden/ by running the GR-Athena++
reference CPU build (oracle/ref, built from the reference sources) on small
cases.  Run from the repository root:

    make -C oracle/ref -j8          # needs the reference checkout
    python tests/golden/make_golden.py [ops_<case> evol_<case> ...]

Fixtures (numpy .npz, compressed):
  ops_<case>.npz    one Mesh after initialisation ("u0") and the reference's
                    output of every operator on it plus every stage of one
                    time step (records written by oracle/ref/z4c_ops_driver.cpp)
  evol_<case>.npz   a multi-step run of the stock reference driver: the
                    history table (outputs/history.cpp columns) and the
                    initial and final states
  weyl_punc2.npz    Z4cWeyl (Re, Im psi4) on the initial state of ops_punc2
                    and after its one RK4 step; psi4 extraction (ghost
                    exchange of the Weyl register, sphere interpolation and
                    (l, m) projection) of the latter
  restart_ml.npz    the reference's restart file after one step on the
                    two-level mesh of ml_exchange_outflow, without its
                    MeshBlock data
  restart_track4.npz  the reference's restart file of the evol_track4 run
                    without its MeshBlock data (that is evol_track4's final
                    state)
  refine_vc.npz     the vertex-centred restriction and prolongation operators
                    of one MeshBlock of a statically refined mesh, and the
                    regrid-time state transfer (coarse to fine, fine to
                    coarse) between two of its blocks
  amr_<case>.npz    an adaptive run of the stock reference driver: MeshBlock
                    lists, dt and puncture-tracker positions of every cycle,
                    the history table, sums and samples of the initial and
                    final states
  ml_exchange_<bc>.npz  one vertex-centred ghost fill of a two-level mesh
                    (restriction, additive unpack with node multiplicity,
                    coarse-level BCs, prolongation, fine-level BCs) of an
                    integer-hash state (ml_hash_state), outflow and periodic
                    faces, with the MeshBlocks' logical locations and
                    coordinates
Each fixture stores the input-deck parameters it was made with ("params",
"mesh", "integrator" as JSON strings).
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
sys.path.insert(0, HERE)
from z4cio import read_records  # noqa: E402

OPS_KEEP = ["meta", "xf", "xv", "dx", "time_dt", "u0", "rhs0", "alg0", "adm0", "con0",
            "uadm0", "gx_pre", "gx_post", "s1_rhs", "s1_alg", "s2_alg", "s3_alg", "s4_alg",
            "s4_adm", "s4_con"]

# run-time options of the cases (reference <z4c> block); r_max_con is always
# given explicitly: the reference turns its +inf default into 0 on every
# MeshBlock after the first (parameter_input.cpp:129-135, 732-752).
GAUGE_WAVE = dict(lapse_harmonic=1.0, lapse_harmonicf=0.0, lapse_oplog=0.0,
                  lapse_advect=0.0, shift_Gamma=0.0, shift_eta=0.0, shift_advect=0.0,
                  diss=0.02, damp_kappa1=0.02, damp_kappa2=0.0, r_max_con=1e300)
PUNCTURE = dict(diss=0.02, chi_div_floor=1e-5, damp_kappa1=0.02, damp_kappa2=0.0,
                shift_eta=2.0, r_max_con=1e300)

CASES = {
    # the gauge-wave benchmark's physics on one 8^3 block (periodic)
    "gw1": dict(test="gauge_wave1", z4c=GAUGE_WAVE, integ="rk4", bc="periodic",
                mesh=[(8, -0.5, 0.5, 8)] * 3, extra={"AwA_amplitude": 0.01}),
    # one puncture, two blocks along x, outflow faces (the puncture benchmark's gauge)
    "punc2": dict(test="one_puncture", z4c=PUNCTURE, integ="rk4", bc="extrapolate_outflow",
                  mesh=[(16, -4.0, 4.0, 8), (8, -2.0, 2.0, 8), (8, -2.0, 2.0, 8)],
                  extra={}, problem={"punc_ADM_mass": 1.0}),
    # the reference's robust-stability noise, two periodic blocks, Butcher RK4
    "rs2": dict(test="robust_stability", z4c=PUNCTURE, integ="bt_rk4", bc="periodic",
                mesh=[(16, -4.0, 4.0, 8), (8, -2.0, 2.0, 8), (8, -2.0, 2.0, 8)],
                extra={"AwA_amplitude": 1e-10}),
    # one puncture, two blocks along x, gr_sommerfeld faces (Z4cBoundaryRHS)
    "somm2": dict(test="one_puncture", z4c=PUNCTURE, integ="rk4", bc="gr_sommerfeld",
                  mesh=[(16, -4.0, 4.0, 8), (8, -2.0, 2.0, 8), (8, -2.0, 2.0, 8)],
                  extra={}, problem={"punc_ADM_mass": 1.0}),
}
# records every ops fixture keeps when the driver wrote them
OPS_OPTIONAL = ["brhs0"]

EVOL = {
    # the benchmark gauge wave, one 16^3 block, 40 steps, history every step
    "gw16": dict(test="gauge_wave1", z4c=GAUGE_WAVE, integ="rk4", bc="periodic",
                 mesh=[(16, -0.5, 0.5, 16)] * 3, extra={"AwA_amplitude": 0.01}, nlim=40),
    # one puncture on 2x2x1 blocks with outflow boundaries, 12 steps
    "punc4": dict(test="one_puncture", z4c=PUNCTURE, integ="rk4", bc="extrapolate_outflow",
                  mesh=[(16, -4.0, 4.0, 8), (16, -4.0, 4.0, 8), (8, -2.0, 2.0, 8)], extra={},
                  problem={"punc_ADM_mass": 1.0}, nlim=12),
    # the same puncture with gr_sommerfeld faces, 8 steps
    "somm4": dict(test="one_puncture", z4c=PUNCTURE, integ="rk4", bc="gr_sommerfeld",
                  mesh=[(16, -4.0, 4.0, 8), (16, -4.0, 4.0, 8), (8, -2.0, 2.0, 8)], extra={},
                  problem={"punc_ADM_mass": 1.0}, nlim=8),
    # the puncture of punc4 with a puncture tracker started off the origin
    # (z4c/puncture_tracker.cpp), 10 steps; the tracker file is recorded
    "track4": dict(test="one_puncture", z4c=PUNCTURE, integ="rk4", bc="extrapolate_outflow",
                   mesh=[(16, -4.0, 4.0, 8), (16, -4.0, 4.0, 8), (8, -2.0, 2.0, 8)],
                   extra={"npunct": 1, "bh_0_x": 0.37, "bh_0_y": -0.21, "bh_0_z": 0.13},
                   problem={"punc_ADM_mass": 1.0}, nlim=10, tracker=True),
}
# The benchmark configurations at their stated sizes and lengths.  Their
# states are too large to store (1.4 GB per register on the 512-block mesh),
# so a fixture keeps the history table of every step, per-variable sums of
# the initial and final states, and a strided sample of the final state on a
# few MeshBlocks; the test regenerates the initial state on its side.
SCALE = {
    # the gauge-wave benchmark as written: 48^3 cells in one periodic block, harmonic-like
    # lapse, zero shift, A = 0.01, KO 0.02, kappa1 0.02, 1000 rk4 steps
    "gw48": dict(test="gauge_wave1", z4c=GAUGE_WAVE, integ="rk4", bc="periodic",
                 mesh=[(48, -0.5, 0.5, 48)] * 3, extra={"AwA_amplitude": 0.01}, nlim=1000,
                 stride=4, sample_blocks=[0]),
    # the single-puncture benchmark: M = 1 at the origin, pre-collapsed lapse,
    # 128^3 cells as 512 blocks of 16^3 on [-16, 16]^3, outflow faces
    "punc512": dict(test="one_puncture", z4c=PUNCTURE, integ="rk4", bc="extrapolate_outflow",
                    mesh=[(128, -16.0, 16.0, 16)] * 3, extra={},
                    problem={"punc_ADM_mass": 1.0}, nlim=40, stride=2,
                    sample_blocks=[0, 73, 219, 292, 365, 511]),
    # the robust-stability benchmark: Minkowski plus U(-1e-10, 1e-10) on all 22
    # Z4c variables at every vertex (initial_data.noise_state, seed 137),
    # periodic, injected into the reference
    "rs512": dict(test="inject", z4c=PUNCTURE, integ="rk4", bc="periodic",
                  mesh=[(128, -16.0, 16.0, 16)] * 3, extra={}, nlim=40, stride=2,
                  noise=dict(amplitude=1e-10, seed=137), sample_blocks=[0, 73, 219, 292, 365, 511]),
}
BC_CODES = {"periodic": 0, "extrapolate_outflow": 1, "gr_sommerfeld": 2}

# An adaptive run in the manner of the adaptive binary benchmark, small: Brill-Lindquist
# punctures (m = 0.5 each, a fraction of a cell off (+-1.5, 0, 0)) on
# [-8, 8]^3 with 2^3 root MeshBlocks of 8^3, 4 levels, refined by the
# reference's Linf_box_in_box criterion around the two puncture trackers
# (par_b = 1.5), derefinement after 3 flagged cycles.  A constant initial
# shift beta^x = -1 with a weak Gamma-driver damping (eta = 0.5) carries the
# trackers across the refinement boundaries: the run refines at cycle 17 and
# derefines at cycle 44 of its 60.
AMR = {
    "bbh_amr": dict(test="brill_lindquist", z4c=dict(PUNCTURE, shift_eta=0.5), integ="rk4",
                    bc="extrapolate_outflow", mesh=[(16, -8.0, 8.0, 8)] * 3,
                    amr=dict(numlevel=4, derefine_count=3),
                    extra={"npunct": 2,
                           "bh_0_x": 1.5 + 0.0625 * 0.37, "bh_0_y": 0.0625 * 0.21,
                           "bh_0_z": 0.0625 * 0.13,
                           "bh_1_x": -1.5 - 0.0625 * 0.37, "bh_1_y": -0.0625 * 0.21,
                           "bh_1_z": -0.0625 * 0.13},
                    problem={"bl_m_0": 0.5, "bl_m_1": 0.5, "par_b": 1.5, "shift_x": -1.0},
                    nlim=60, stride=2, tracker=True),
}


def deck(case, out_file, nlim=1, dump_initial="", dump_final="", hst=False, threads=1):
    lines = ["<job>", "problem_id = golden", "<z4c>"]
    for k, v in {**case["z4c"], **case.get("extra", {})}.items():
        lines.append(f"{k} = {v!r}" if isinstance(v, float) else f"{k} = {v}")
    lines += ["<task_triggers>", "adjust_mesh_dt = false",
              "<time>", "cfl_number = 0.25", "tlim = 1e10", f"nlim = {nlim}",
              f"integrator = {case['integ']}", "ncycle_out = 1000000", "<mesh>"]
    for a, (nx, lo, hi, _) in enumerate(case["mesh"]):
        d = a + 1
        lines += [f"nx{d} = {nx}", f"x{d}min = {lo!r}", f"x{d}max = {hi!r}",
                  f"ix{d}_bc = {case['bc']}", f"ox{d}_bc = {case['bc']}"]
    amr = case.get("amr")
    if amr:
        lines += ["refinement = adaptive", f"numlevel = {amr['numlevel']}",
                  f"derefine_count = {amr['derefine_count']}"]
    else:
        lines.append("refinement = none")
    lines += [f"num_threads = {threads}", "<meshblock>"]
    for a, (_, _, _, nb) in enumerate(case["mesh"]):
        lines.append(f"nx{a + 1} = {nb}")
    lines += ["<problem>", f"test = {case['test']}"]
    for k, v in case.get("problem", {}).items():
        lines.append(f"{k} = {v}")
    if dump_initial:
        lines.append(f"dump_initial = {dump_initial}")
    if dump_final:
        lines.append(f"dump_final = {dump_final}")
    lines += ["<driver>", f"out = {out_file}"]
    if hst:
        lines += ["<output1>", "file_type = hst", "dt = 1e-12", "data_format = %.17e"]
    if case.get("tracker"):
        lines[lines.index("<task_triggers>") + 1:lines.index("<task_triggers>") + 1] = [
            "dt_Z4c_tracker_punctures = 1e-12"]
    return "\n".join(lines) + "\n"


def meta_json(case):
    nb = [m[0] // m[3] for m in case["mesh"]]
    nx = [m[3] for m in case["mesh"]]
    bc = BC_CODES[case["bc"]]
    mesh = dict(nb=nb, nx=nx, xmin=[m[1] for m in case["mesh"]],
                xmax=[m[2] for m in case["mesh"]], bc=[bc] * 6)
    return dict(params=json.dumps(case["z4c"]), mesh=json.dumps(mesh),
                integrator=json.dumps(case["integ"]))


def make_ops(name, case, outdir):
    with tempfile.TemporaryDirectory() as tmp:
        rec_path = os.path.join(tmp, "ops.rec")
        inp = os.path.join(tmp, "case.inp")
        with open(inp, "w") as f:
            f.write(deck(case, rec_path))
        subprocess.run([os.path.join(REF_BIN, "z4c_ops_ref"), "-i", inp], cwd=tmp, check=True,
                       stdout=subprocess.DEVNULL)
        rec = read_records(rec_path)
    out = {k: rec[k] for k in OPS_KEEP}
    out.update({k: rec[k] for k in OPS_OPTIONAL if k in rec})
    out.update(meta_json(case))
    path = os.path.join(outdir, f"ops_{name}.npz")
    np.savez_compressed(path, **out)
    return path


def parse_hst(path):
    rows = []
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                continue
            rows.append([float(x) for x in line.split()])
    return np.array(rows)


def make_evol(name, case, outdir):
    with tempfile.TemporaryDirectory() as tmp:
        inp = os.path.join(tmp, "case.inp")
        init, final = os.path.join(tmp, "init.rec"), os.path.join(tmp, "final.rec")
        with open(inp, "w") as f:
            f.write(deck(case, "unused", nlim=case["nlim"], dump_initial=init,
                         dump_final=final, hst=True))
        subprocess.run([os.path.join(REF_BIN, "athena_ref"), "-i", inp], cwd=tmp, check=True,
                       stdout=subprocess.DEVNULL)
        hst = parse_hst(os.path.join(tmp, "golden.hst"))
        r0, r1 = read_records(init), read_records(final)
        track = None
        if case.get("tracker"):  # 1:iter 2:time 3:x 4:y 5:z 6:betax 7:betay 8:betaz
            track = np.loadtxt(os.path.join(tmp, "golden.puncture_0.txt"), ndmin=2)
    out = dict(hst=hst, meta=r0["meta"], xf=r0["xf"], xv=r0["xv"], dx=r0["dx"],
               time_dt=r1["time_dt"], u_init=r0["u"], u_final=r1["u"],
               con_final=r1["con"], nlim=np.array(case["nlim"]))
    if track is not None:
        out["tracker"] = track
        out["tracker_start"] = np.array([case["extra"][f"bh_0_{c}"] for c in "xyz"])
    out.update(meta_json(case))
    path = os.path.join(outdir, f"evol_{name}.npz")
    np.savez_compressed(path, **out)
    return path


def gid_order(nb):
    """Grid index l0 + nb0 (l1 + nb1 l2) of every MeshBlock of a uniform
    block grid, in gid order: the leaves of the root tree in Morton order
    with x the lowest bit."""
    def morton(l):
        key = 0
        for bit in range(16):
            for a in range(3):
                key |= ((l[a] >> bit) & 1) << (3 * bit + a)
        return key
    locs = [(i, j, k) for k in range(nb[2]) for j in range(nb[1]) for i in range(nb[0])]
    return [l[0] + nb[0] * (l[1] + nb[1] * l[2]) for l in sorted(locs, key=morton)]


def state_sums(u):
    """Per-variable sum, sum of squares and largest magnitude over the
    interior vertices of every block of a [block][var][k][j][i] state."""
    I = u[:, :, NG_:-NG_, NG_:-NG_, NG_:-NG_]
    return np.stack([I.sum(axis=(0, 2, 3, 4)), (I * I).sum(axis=(0, 2, 3, 4)),
                     np.abs(I).max(axis=(0, 2, 3, 4))], axis=1)


NG_ = 4


def noise_state_gid(case):
    """The robust-stability state of a SCALE case in gid order (the package's
    seeded generator, grid order, reordered)."""
    sys.path.insert(0, os.path.join(ROOT, "gr-athena_b200"))
    import z4c_b200 as Z
    from z4c_b200 import initial_data as ID
    nb = [m[0] // m[3] for m in case["mesh"]]
    mesh = Z.Mesh(nb, [m[3] for m in case["mesh"]], [m[1] for m in case["mesh"]],
                  [m[2] for m in case["mesh"]], case["bc"])
    u = ID.noise_state(mesh, **case["noise"])
    return u[gid_order(nb)]


def make_scale(name, case, outdir, threads=None):
    threads = threads or os.cpu_count()
    with tempfile.TemporaryDirectory() as tmp:
        inp = os.path.join(tmp, "case.inp")
        init, final = os.path.join(tmp, "init.rec"), os.path.join(tmp, "final.rec")
        text = deck(case, "unused", nlim=case["nlim"], dump_initial=init, dump_final=final,
                    hst=True, threads=threads)
        if case["test"] == "inject":
            from z4cio import write_records
            inj = os.path.join(tmp, "inject.rec")
            write_records(inj, {"u": noise_state_gid(case)})
            text = text.replace("<driver>", f"inject_file = {inj}\n<driver>")
        with open(inp, "w") as f:
            f.write(text)
        subprocess.run([os.path.join(REF_BIN, "athena_ref"), "-i", inp], cwd=tmp, check=True,
                       stdout=subprocess.DEVNULL)
        hst = parse_hst(os.path.join(tmp, "golden.hst"))
        r0 = read_records(init)
        u_init_sums = state_sums(r0["u"])
        meta = r0["meta"]
        del r0
        r1 = read_records(final)
    nb = [m[0] // m[3] for m in case["mesh"]]
    order = [int(m[2] + nb[0] * (m[3] + nb[1] * m[4])) for m in meta]
    assert order == gid_order(nb), "gid order"
    s = case["stride"]
    blocks = case["sample_blocks"]  # grid indices
    gids = [order.index(b) for b in blocks]
    sub = r1["u"][gids][:, :, ::s, ::s, ::s]
    out = dict(hst=hst, meta=meta, time_dt=r1["time_dt"], nlim=np.array(case["nlim"]),
               u_init_sums=u_init_sums, u_final_sums=state_sums(r1["u"]),
               con_final_sums=state_sums(r1["con"]), sample_blocks=np.array(blocks),
               stride=np.array(s), u_final_sample=sub, threads=np.array(threads))
    if "noise" in case:
        out["noise"] = json.dumps(case["noise"])
    out.update(meta_json(case))
    path = os.path.join(outdir, f"scale_{name}.npz")
    np.savez_compressed(path, **out)
    return path


def make_amr(name, case, outdir, threads=None):
    """The stock reference driver on an adaptive mesh (AMR cases): the
    MeshBlock list, time, dt and puncture-tracker positions at the top of
    every cycle (the oracle problem generator's dump_blocks), the history
    table, and sums plus a strided sample (four MeshBlocks) of the initial
    and final states."""
    threads = threads or os.cpu_count()
    with tempfile.TemporaryDirectory() as tmp:
        inp = os.path.join(tmp, "case.inp")
        init, final = os.path.join(tmp, "init.rec"), os.path.join(tmp, "final.rec")
        blocks = os.path.join(tmp, "blocks.rec")
        text = deck(case, "unused", nlim=case["nlim"], dump_initial=init, dump_final=final,
                    hst=True, threads=threads)
        text = text.replace("<driver>", f"dump_blocks = {blocks}\n<driver>")
        with open(inp, "w") as f:
            f.write(text)
        subprocess.run([os.path.join(REF_BIN, "athena_ref"), "-i", inp], cwd=tmp, check=True,
                       stdout=subprocess.DEVNULL)
        hst = parse_hst(os.path.join(tmp, "golden.hst"))
        rb = read_records(blocks)
        s = case["stride"]
        out = dict(hst=hst, blocks=rb["blocks"], cycles=rb["cycles"], trackers=rb["trackers"],
                   nlim=np.array(case["nlim"]), stride=np.array(s), threads=np.array(threads))
        for tag, path in (("init", init), ("final", final)):
            r = read_records(path)
            nb = r["u"].shape[0]
            pick = np.array(sorted({0, nb // 3, (2 * nb) // 3, nb - 1}))
            out[f"{tag}_meta"] = r["meta"]
            out[f"{tag}_sample_blocks"] = pick
            out[f"u_{tag}_sample"] = r["u"][pick][:, :, ::s, ::s, ::s]
            out[f"u_{tag}_sums"] = state_sums(r["u"])
            if tag == "final":
                out["con_final_sums"] = state_sums(r["con"])
                out["time_dt"] = r["time_dt"]
            del r
    out.update(meta_json(case))
    out["amr"] = json.dumps(case["amr"])
    out["extra"] = json.dumps(case["extra"])
    out["problem"] = json.dumps(case["problem"])
    path = os.path.join(outdir, f"amr_{name}.npz")
    np.savez_compressed(path, **out)
    return path


# vertex-centred refinement operators (mesh/mesh_refinement_vc.cpp) on one
# MeshBlock of a statically refined mesh: 16^3 cells as 2^3 blocks of 8^3 at
# the root level, the centre refined once
REFINE = dict(test="one_puncture", z4c=PUNCTURE, integ="rk4", bc="extrapolate_outflow",
              mesh=[(16, -4.0, 4.0, 8)] * 3, extra={}, problem={"punc_ADM_mass": 1.0})


# psi4 extraction spheres of the Weyl fixture (<psi4_extraction> block): one
# sphere inside the domain of ops_punc2 and one that leaves it through the y
# and z faces
WAVE = dict(num_radii=2, radius_0=1.5, radius_1=3.0, nlev=6, lmax=4)
WAVE_DECK = "<psi4_extraction>\n" + "".join(f"{k} = {v}\n" for k, v in WAVE.items())


def make_weyl(outdir):
    """Z4cWeyl on the initial state of the ops_punc2 case and after its one
    RK4 step (the inputs, u0/adm0 and s4_alg/s4_adm, are in ops_punc2.npz),
    and the psi4 multipoles of the second on the WAVE spheres; only the Weyl
    and extraction records are stored."""
    with tempfile.TemporaryDirectory() as tmp:
        rec_path = os.path.join(tmp, "ops.rec")
        inp = os.path.join(tmp, "case.inp")
        with open(inp, "w") as f:
            f.write(deck(CASES["punc2"], rec_path) + "weyl = true\n" + WAVE_DECK)
        subprocess.run([os.path.join(REF_BIN, "z4c_ops_ref"), "-i", inp], cwd=tmp, check=True,
                       stdout=subprocess.DEVNULL)
        rec = read_records(rec_path)
    path = os.path.join(outdir, "weyl_punc2.npz")
    # weyl0 on the initial data (K_ab = 0), weyl1 after one RK4 step (K_ab
    # nonzero); a corner of each input state ties them to ops_punc2
    wave = {k[len("s4_wave_"):]: v for k, v in rec.items() if k.startswith("s4_wave_")}
    np.savez_compressed(path, weyl0=rec["weyl0"], weyl1=rec["s4_weyl"],
                        u0=rec["u0"][:, :1, :1, :1, :1],
                        s4_alg=rec["s4_alg"][:, :1, :1, :1, :1],
                        wave=json.dumps(WAVE), **{"wave_" + k: v for k, v in wave.items()})
    return path


def make_refine(outdir):
    with tempfile.TemporaryDirectory() as tmp:
        rec_path = os.path.join(tmp, "refine.rec")
        inp = os.path.join(tmp, "case.inp")
        text = deck(REFINE, rec_path).replace("refinement = none", "refinement = static")
        text += "refine_ops_only = true\n<refinement1>\n" + "".join(
            f"x{d}min = -0.5\nx{d}max = 0.5\n" for d in (1, 2, 3)) + "level = 1\n"
        with open(inp, "w") as f:
            f.write(text)
        subprocess.run([os.path.join(REF_BIN, "z4c_ops_ref"), "-i", inp], cwd=tmp, check=True,
                       stdout=subprocess.DEVNULL)
        rec = read_records(rec_path)
    # the operators act on every variable alike: keep three of them
    keep = [0, 7, 21]
    out = {k: (v if v.ndim == 1 else v[keep]) for k, v in rec.items()
           if k.startswith("rf_") or k.startswith("rg_")}
    out["nx"] = np.array([8, 8, 8])
    path = os.path.join(outdir, "refine_vc.npz")
    np.savez_compressed(path, **out)
    return path


# multilevel ghost exchange: the 16^3-cell mesh of REFINE with one root
# block (x > 0, y < 0, z < 0) refined once, so that its eight children sit
# between coarse blocks in gid order; outflow and periodic faces
ML_REGION = dict(x1min=0.5, x1max=3.5, x2min=-3.5, x2max=-0.5, x3min=-3.5, x3max=-0.5, level=1)
ML_VARS = [0, 13]


def ml_hash_state(nblocks, nvar, nn):
    """The integer-hash state the operator driver's gx_hash option writes."""
    g, n, k, j, i = np.meshgrid(np.arange(nblocks), np.arange(nvar), np.arange(nn),
                                np.arange(nn), np.arange(nn), indexing="ij")
    return ((g * 131 + n * 31 + k * 7 + j * 3 + i) % 1009) / 1009.0 - 0.5


def make_multilevel(bc, outdir):
    case = dict(REFINE, bc=bc)
    with tempfile.TemporaryDirectory() as tmp:
        rec_path = os.path.join(tmp, "ml.rec")
        inp = os.path.join(tmp, "case.inp")
        text = deck(case, rec_path).replace("refinement = none", "refinement = static")
        text += "gx_hash = true\n<refinement1>\n" + "".join(
            f"{k} = {v}\n" for k, v in ML_REGION.items())
        with open(inp, "w") as f:
            f.write(text)
        subprocess.run([os.path.join(REF_BIN, "z4c_ops_ref"), "-i", inp], cwd=tmp, check=True,
                       stdout=subprocess.DEVNULL)
        rec = read_records(rec_path)
    pre = rec["gx_pre"]
    assert np.array_equal(pre, ml_hash_state(*pre.shape[:2], pre.shape[2])), "gx_hash state"
    tag = {"extrapolate_outflow": "outflow", "periodic": "periodic"}[bc]
    path = os.path.join(outdir, f"ml_exchange_{tag}.npz")
    np.savez_compressed(path, gx_post=rec["gx_post"][:, ML_VARS], vars=np.array(ML_VARS),
                        meta=rec["meta"], xf=rec["xf"], dx=rec["dx"], bc=BC_CODES[bc], nb=np.array([2, 2, 2]),
                        nx=np.array([8, 8, 8]), xmin=np.array([-4.0] * 3), xmax=np.array([4.0] * 3),
                        region=json.dumps(ML_REGION))
    return path


RST_DECK = "<output2>\nfile_type = rst\ndt = 1e10\n"


def make_restart(outdir):
    """The restart file the stock reference driver writes at the end of the
    evol_track4 run (<output2> file_type = rst): everything before the
    MeshBlock data (parameter text, header, the tracker record, ID list) is
    stored; the data section is the run's final state, which evol_track4.npz
    already holds (checked here), so the test rebuilds the file byte for
    byte."""
    case = EVOL["track4"]
    with tempfile.TemporaryDirectory() as tmp:
        inp = os.path.join(tmp, "case.inp")
        final = os.path.join(tmp, "final.rec")
        with open(inp, "w") as f:
            f.write(deck(case, "unused", nlim=case["nlim"], dump_final=final) + RST_DECK)
        subprocess.run([os.path.join(REF_BIN, "athena_ref"), "-i", inp], cwd=tmp, check=True,
                       stdout=subprocess.DEVNULL)
        raw = open(os.path.join(tmp, "golden.final.rst"), "rb").read()
        u = read_records(final)["u"]
    data = u.astype("<f8").tobytes()
    assert raw.endswith(data), "restart data section is not the final state in gid order"
    ev = np.load(os.path.join(outdir, "evol_track4.npz"))
    assert np.array_equal(ev["u_final"], u), "evol_track4 fixture is stale"
    prefix = np.frombuffer(raw[:len(raw) - len(data)], dtype=np.uint8)
    path = os.path.join(outdir, "restart_track4.npz")
    np.savez_compressed(path, prefix=prefix, rst_deck=RST_DECK)
    return path


def make_restart_ml(outdir):
    """The restart file the stock reference driver writes after one step
    on the outflow two-level mesh of ml_exchange_outflow: everything before
    the MeshBlock data (parameter text, header, ID list with the blocks'
    levels) is stored."""
    case = dict(REFINE, bc="extrapolate_outflow")
    with tempfile.TemporaryDirectory() as tmp:
        inp = os.path.join(tmp, "case.inp")
        text = deck(case, "unused", nlim=1).replace("refinement = none", "refinement = static")
        text += RST_DECK + "<refinement1>\n" + "".join(f"{k} = {v}\n" for k, v in ML_REGION.items())
        with open(inp, "w") as f:
            f.write(text)
        subprocess.run([os.path.join(REF_BIN, "athena_ref"), "-i", inp], cwd=tmp, check=True,
                       stdout=subprocess.DEVNULL)
        raw = open(os.path.join(tmp, "golden.final.rst"), "rb").read()
    nbytes = 15 * 22 * 17 ** 3 * 8
    prefix = np.frombuffer(raw[:len(raw) - nbytes], dtype=np.uint8)
    path = os.path.join(outdir, "restart_ml.npz")
    np.savez_compressed(path, prefix=prefix, data_bytes=nbytes)
    return path


def main():
    only = set(sys.argv[1:])  # fixture names to (re)make; all when empty
    if not only or "weyl_punc2" in only:
        p = make_weyl(HERE)
        print(f"{p}: {os.path.getsize(p) / 1e6:.2f} MB")
    if not only or "refine_vc" in only:
        p = make_refine(HERE)
        print(f"{p}: {os.path.getsize(p) / 1e6:.2f} MB")
    for name, case in CASES.items():
        if only and f"ops_{name}" not in only:
            continue
        p = make_ops(name, case, HERE)
        print(f"{p}: {os.path.getsize(p) / 1e6:.2f} MB")
    for name, case in EVOL.items():
        if only and f"evol_{name}" not in only:
            continue
        p = make_evol(name, case, HERE)
        print(f"{p}: {os.path.getsize(p) / 1e6:.2f} MB")
    for bc in ("extrapolate_outflow", "periodic"):
        tag = {"extrapolate_outflow": "outflow", "periodic": "periodic"}[bc]
        if not only or f"ml_exchange_{tag}" in only:
            p = make_multilevel(bc, HERE)
            print(f"{p}: {os.path.getsize(p) / 1e6:.2f} MB")
    if not only or "restart_ml" in only:
        p = make_restart_ml(HERE)
        print(f"{p}: {os.path.getsize(p) / 1e6:.2f} MB")
    if not only or "restart_track4" in only:  # needs evol_track4
        p = make_restart(HERE)
        print(f"{p}: {os.path.getsize(p) / 1e6:.2f} MB")
    for name, case in AMR.items():
        if only and f"amr_{name}" not in only:
            continue
        p = make_amr(name, case, HERE)
        print(f"{p}: {os.path.getsize(p) / 1e6:.2f} MB")
    for name, case in SCALE.items():  # minutes each: the reference at full size
        if only and f"scale_{name}" not in only:
            continue
        p = make_scale(name, case, HERE)
        print(f"{p}: {os.path.getsize(p) / 1e6:.2f} MB")


if __name__ == "__main__":
    main()
