"""WAVEGUIDE_STRAIGHT, WAVEGUIDE_PML and WAVEGUIDE_IRIS: WR90 guides
(2 x 46 x 100 cells) driven by a TE10 mode excitation read from a mode file
(Excitation_mode_list, mode_excitation.F90), ended by mode-impedance thin
layers or a PML, sampled by mode outputs (Output_mode_list,
output_modes.F90) and carried through each case's own post-processing input:

* STRAIGHT: four mode outputs Fourier transformed (option 3), then the
  one-port analysis (option 9): waveguide_straight.fout_ref byte for byte;
  the run's .field.tout byte for byte and its .mode.tout line for line but
  for round-off-level values (the reference's FP64 sums differ in the last
  bits: its 1e-14 residues where the field is still zero, and one 7th digit);
* PML: Ex1.tout_ref (option 1 on the mode file) and waveguide_pml.fout_ref
  (options 3 and 9) byte for byte;
* IRIS: PEC blocks whose outer faces lie on the mesh boundary, where connect
  never runs (connect.F90:180-213), eight mode outputs and the two-port
  analysis (option 10): waveguide_iris.fout_ref byte for byte, the field
  file to its E16.7 digits.

GPU: the library against the oracle on the same tables, and the straight
case through the runner and the post-processor CLIs."""
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import inp, post_process
from ggi_tlm_b200 import run as runner
from ggi_tlm_b200.problem import build_tables

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import test_inp as T  # noqa: E402
import test_thin_layer as TL  # noqa: E402
import oracle  # noqa: E402

CASES = ["waveguide_straight", "waveguide_pml", "waveguide_iris"]


def opener(case):
    data = np.load(os.path.join(HERE, "golden", "data_text.npz"))
    return lambda name: [str(x) for x in data[name.strip() + "@" + case]]


def problem(case, lines=None):
    p = inp.read_inp(lines or T.inputs()[case], T.materials, open_file=opener(case), thin_layer=TL.thin_layer)
    return p, build_tables(p.spec)


def text(npz, key):
    return [str(x) for x in np.load(os.path.join(HERE, "golden", npz + ".npz"))[key]]


def post_lines(case):
    """The case's post-processing input up to its visualisation options (17,
    5: animations), which end it here."""
    post = text("post_process_text", case)
    stop = [i for i, x in enumerate(post) if x.split()[:1] in (["17"], ["5"]) and "OPTION" in x.upper()]
    return post[:stop[0]] + ["0"] if stop else post


def oracle_run(t, spec):
    o = oracle.Oracle(t, threads=min(8, os.cpu_count() or 1))
    n = int(t["n_timesteps"])
    cell = o.run(n)
    face = o.face_probes() if int(t["n_face_probes"]) else np.zeros((0, n))
    dft = o.dft() if spec.dft_surfaces else None
    o.close()
    return cell, face, dft, oracle.mode_outputs(t)


def test_reader_takes_the_mode_file():
    p, t = problem("waveguide_straight")
    mode = [ln.split() for ln in opener("waveguide_straight")("WR90.mode")]
    ex = p.spec.point_excitations
    # 92 samples in the mode file's order, moved onto the excitation plane (z = -0.0125: the faces
    # between cells 25 and 26, the zplane's faces seen from cell 26 as the side is -1), weighted by
    # column 6
    assert len(ex) == len(mode) == 92
    assert [e.cell[:2] for e in ex] == [(int(m[0]), int(m[1])) for m in mode]
    assert all(e.cell[2] == 26 and e.face == "zmin" and e.one_side for e in ex)
    assert [e.scale for e in ex] == [float(m[5]) for m in mode]
    assert np.array_equal(t["fpt_side"], np.full(92, 1))
    # the first output mode on the plane z = -0.0005, side 1: the max faces of the cells below
    assert {(c[2], code) for c, code, _ in p.spec.mode_outputs[0].samples} == {(49, 6)}
    # four mode outputs, each on its plane's own side
    assert [len(m.samples) for m in p.spec.mode_outputs] == [92] * 4
    assert int(t["n_modes"]) == 4 and np.array_equal(t["mode_field"][:92], [float(m[5]) for m in mode])
    # side 0: the faces as for -1, each side half the mode field
    lines = list(T.inputs()["waveguide_straight"])
    k = next(i for i, x in enumerate(lines) if x.lower().startswith("excitation_mode_list"))
    lines[k + 5] = "0"
    p0, t0 = problem("waveguide_straight", lines)
    assert [e.scale for e in p0.spec.point_excitations] == [float(m[5]) / 2.0 for m in mode]
    assert np.array_equal(t0["fpt_side"], np.zeros(92))


def test_a_mode_file_that_does_not_fit_its_surface_is_refused():
    lines = list(T.inputs()["waveguide_straight"])
    short = opener("waveguide_straight")("WR90.mode")[:-2]  # one row of the cross section missing
    with pytest.raises(ValueError, match="extent"):
        inp.read_inp(lines, T.materials, open_file=lambda name: short, thin_layer=TL.thin_layer)


@pytest.mark.parametrize("case", CASES)
def test_oracle_runs_reproduce_the_reference_files(tmp_path, case):
    d = str(tmp_path)
    p, t = problem(case)
    cell, face, dft, modes = oracle_run(t, p.spec)
    runner.write_results(case, p, t, cell, face, None, d, dft=dft, modes=modes)
    post_process.run(post_lines(case), d)
    assert open(os.path.join(d, case + ".fout")).read().splitlines() == text("fout_text", case)
    res = np.load(os.path.join(HERE, "golden", "result_text.npz"))
    if case == "waveguide_pml":
        # option 1 on mode output 1: line for line but for round-off residues where the field is ~0
        got = open(os.path.join(d, "Ex1.tout")).read().splitlines()
        gold = [str(x) for x in res["waveguide_pml_Ex1"]]
        assert got[:3] == gold[:3] and len(got) == len(gold)
        assert sum(a != b for a, b in zip(got, gold)) <= 0.001 * len(gold)
        a, b = np.loadtxt(got[3:]), np.loadtxt(gold[3:])
        assert np.array_equal(a[:, :2], b[:, :2])
        assert np.max(np.abs(a[:, 2] - b[:, 2])) <= 1e-12 * np.abs(b[:, 2]).max()
        return
    got = open(os.path.join(d, case + ".field.tout")).read().splitlines()
    gold = [str(x) for x in res[case + "_field"]]
    assert got[:3] == gold[:3] and len(got) == len(gold)
    if case == "waveguide_straight":
        assert got == gold
        mt = open(os.path.join(d, case + ".mode.tout")).read().splitlines()
        mg = [str(x) for x in res[case + "_mode"]]
        assert len(mt) == len(mg) and sum(a != b for a, b in zip(mt, mg)) <= 5
        a, b = np.loadtxt(mt[3:]), np.loadtxt(mg[3:])
        assert np.array_equal(a[:, :2], b[:, :2])
        assert np.max(np.abs(a[:, 2] - b[:, 2])) <= 1e-6 * np.abs(b[:, 2]).max()
    else:
        assert sum(a == b for a, b in zip(got, gold)) >= 0.99 * len(gold)
        a, b = np.loadtxt(got[3:]), np.loadtxt(gold[3:])
        assert np.max(np.abs(a[:, 2] - b[:, 2])) <= 1e-6 * np.abs(b[:, 2]).max()


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_gpu_mode_waveguides_match_the_oracle(gpu_lib, case):
    from ggi_tlm_b200 import capi

    p, t = problem(case)
    n = int(t["n_timesteps"])
    cell, _, _, modes = oracle_run(t, p.spec)
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(n)
        got_cell, got_modes = g.cell_output(), g.mode_outputs(1, n)
    if cell.size:
        assert np.linalg.norm(got_cell - cell) <= 1e-10 * np.linalg.norm(cell)
    assert np.linalg.norm(got_modes - modes) <= 1e-10 * np.linalg.norm(modes)


@pytest.mark.gpu
def test_gpu_straight_waveguide_through_the_runner_and_the_post_processor(gpu_lib, tmp_path):
    """``python -m ggi_tlm_b200.run waveguide_straight`` in a directory with
    the case's input, mode file and thin-layer file, then the
    post-processor on its own input: the one-port file and the run's
    time-domain files against the reference's (the GPU's FP64 series differ
    from the oracle's by ~1e-13: 99 % of the lines exact, the rest within
    the printed digits)."""
    import subprocess

    d = str(tmp_path)
    case = "waveguide_straight"
    with open(os.path.join(d, case + ".inp"), "w", encoding="latin-1") as f:
        f.write("\n".join(T.inputs()[case]) + "\n")
    with open(os.path.join(d, "WR90.mode"), "w") as f:
        f.write("\n".join(opener(case)("WR90.mode")) + "\n")
    smat = np.load(os.path.join(HERE, "golden", "smat_text.npz"))
    os.makedirs(os.path.join(d, "MATERIAL_DIRECTORY"))
    with open(os.path.join(d, "MATERIAL_DIRECTORY", "WR90_mode_impedance.smat"), "w") as f:
        f.write("\n".join(str(x) for x in smat["WR90_mode_impedance"]) + "\n")
    with open(os.path.join(d, "GGI_TLM_post_process_in.txt"), "w") as f:
        f.write("\n".join(post_lines(case)) + "\n")
    env = dict(os.environ, PYTHONPATH=os.path.dirname(HERE))
    for cmd in (["-m", "ggi_tlm_b200.run", case], ["-m", "ggi_tlm_b200.post_process", "GGI_TLM_post_process_in.txt"]):
        res = subprocess.run([sys.executable, *cmd], cwd=d, env=env, capture_output=True, text=True, timeout=600)
        assert res.returncode == 0, res.stderr[-2000:]
    res = np.load(os.path.join(HERE, "golden", "result_text.npz"))
    for name, gold in ((case + ".fout", text("fout_text", case)),
                       (case + ".field.tout", [str(x) for x in res[case + "_field"]]),
                       (case + ".mode.tout", [str(x) for x in res[case + "_mode"]])):
        got = open(os.path.join(d, name)).read().splitlines()
        assert len(got) == len(gold)
        assert sum(a == b for a, b in zip(got, gold)) >= 0.99 * len(gold)
