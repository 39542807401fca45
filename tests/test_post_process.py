"""The post-processor driven by the reference's own post-processing input
files (ggi_tlm_b200/post_process.py), in a directory holding the run's
result files, as the reference's test cases run it:

* POWER_CALCS: option 3 on the field file and option 15 (transmission cross
  section) with the power surface file give TCS.fout_ref byte for byte (the
  run's files are the case's golden ones);
* PARAMETERISED_FSS: options 1, 3 and 10 on the oracle's run give
  S21.fout_4_ref byte for byte;
* SHIELDING_EFFECTIVENESS_BOX_SLOT: options 3 and 6 on the oracle's run give
  Shielding_effectiveness.fout_ref;
* the answers are read as list-directed reads read them (trailing remarks
  ignored) and unknown options are refused."""
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import inp, post_process, tout
from ggi_tlm_b200 import run as runner
from ggi_tlm_b200.problem import UnsupportedFeature, build_tables

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import test_fss as FSS  # noqa: E402
import test_inp as T  # noqa: E402
import oracle  # noqa: E402


def post_input(name):
    return [str(x) for x in np.load(os.path.join(HERE, "golden", "post_process_text.npz"))[name]]


def fout_golden(name):
    return [str(x) for x in np.load(os.path.join(HERE, "golden", "fout_text.npz"))[name]]


def write_lines(path, lines):
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def test_power_calcs_post_processing_reproduces_tcs(tmp_path):
    d = str(tmp_path)
    g = np.load(os.path.join(HERE, "golden", "power_calc_Ex.npz"))
    n = int(len(g["time"]) / len(np.unique(g["point"])))
    write_lines(os.path.join(d, "power_calc.field.tout"),
                tout.header(len(np.unique(g["point"])), n) +
                [tout.data_line(a, b, c) for a, b, c in zip(g["time"], g["point"], g["value"])])
    write_lines(os.path.join(d, "power_calc.frequency_domain_power_surface.fout"), fout_golden("power_calc"))
    written = post_process.run(post_input("power_calc"), d)
    assert [os.path.basename(x) for x in written] == ["E_field.fout", "TCS.fout"]
    assert open(os.path.join(d, "TCS.fout")).read().splitlines() == fout_golden("power_calc_tcs")


def test_fss_post_processing_reproduces_s21(tmp_path):
    d = str(tmp_path)
    p, t = FSS.problem()
    rows, count = runner._volume_rows(t, p.spec, list(FSS.oracle_averages(t)), "average")
    write_lines(os.path.join(d, "single_cell.volume_average_field.tout"),
                tout.header(count, int(t["n_timesteps"])) + [tout.data_line(a, b, c) for a, b, c in rows])
    written = post_process.run(post_input("fss"), d)
    # eight extractions (option 1), eight transforms (option 3), the two-port analysis (option 10)
    names = [os.path.basename(x) for x in written]
    assert len(names) == 17 and names[:2] == ["Ey1.tout", "Hx1.tout"] and names[-1] == "S21.fout_4"
    assert open(os.path.join(d, "S21.fout_4")).read().splitlines() == fout_golden("fss_s21")


def test_box_slot_post_processing_reproduces_the_shielding_effectiveness(tmp_path):
    d = str(tmp_path)
    p = inp.read_inp(T.inputs()["box_slot"], T.materials)
    t = build_tables(p.spec)
    o = oracle.Oracle(t, threads=os.cpu_count() or 1)
    cell = o.run(int(t["n_timesteps"]))
    o.close()
    runner.write_results("box_slot", p, t, cell, np.zeros((0, int(t["n_timesteps"]))), None, d)
    written = post_process.run(post_input("box_slot"), d)
    assert os.path.basename(written[-1]) == "Shielding_effectiveness.fout"
    got = np.loadtxt(os.path.join(d, "Shielding_effectiveness.fout"), comments="#")
    want = np.loadtxt(fout_golden("box_slot"), comments="#")
    assert got.shape == want.shape
    np.testing.assert_array_equal(got[:, 0], want[:, 0])
    # the spectra's ratio, to the golden file's 7 digits
    np.testing.assert_allclose(got[:, 4], want[:, 4], rtol=2e-6)


def test_answers_and_refusals(tmp_path):
    a = post_process._Answers(["", "  3  POST PROCESSING OPTION", "1e6 fmin", " 1.0D3", "lin"])
    assert a.integer() == 3 and a.number() == 1e6 and a.number() == 1e3 and a.word() == "lin"
    with pytest.raises(UnsupportedFeature, match="option 42"):
        post_process.run(["42"], str(tmp_path))
    assert post_process.run(["0", "3"], str(tmp_path)) == []
