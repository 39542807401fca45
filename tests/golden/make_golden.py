"""Extract the reference's own golden time series for the in-scope
known-answer cases into compact fixtures (tests/golden/*.npz).

Reads GGI_TLM's TEST_DATA/*/PROBLEM_SPECIFICATION_FILES/*.tout_ref (text,
format (E16.7,I5,E16.7), SRC/TLM_MODULES/File_information.F90:235) from the
reference checkout named on the command line (or by the GGI_TLM_REFERENCE
environment variable) and stores (time, value) arrays.  Run once where the reference is present; the
fixtures travel with the repository.

    python tests/golden/make_golden.py /path/to/reference
"""
import os
import sys

import numpy as np

CASES = {
    "tem_pml_Ey": "TEM_PML_TEST/PROBLEM_SPECIFICATION_FILES/Ey.tout_ref",
    "tem_material_Ey": "TEM_MATERIAL_TEST/PROBLEM_SPECIFICATION_FILES/Ey.tout_ref",
    "material_stability_Ey": "MATERIAL_STABILITY_TEST/PROBLEM_SPECIFICATION_FILES/cavity.field.tout_ref",
    "material_test2_Ex": "MATERIAL_TEST2/PROBLEM_SPECIFICATION_FILES/mat_test.field.tout_ref",
    **{f"huygens_box_{f}": f"HUYGENS_SURFACE/PROBLEM_SPECIFICATION_FILES/{f}_centre.tout_ref"
       for f in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")},
    # the case's create_reference_result copies only this file; its excitation.tout_ref is
    # from another delay (its pulse peaks 4.8 ns later than the input's) and is not used
    "excitation_test_Ex": "EXCITATION_FUNCTION_TEST/PROBLEM_SPECIFICATION_FILES/excitation_test.field.tout_ref",
    "power_calc_Ex": "POWER_CALCS/PROBLEM_SPECIFICATION_FILES/power_calc.field.tout_ref",
    # thin layers (dispersive and anisotropic dispersive surface materials)
    "tem_thin_layer": "TEM_THIN_LAYER_TEST/PROBLEM_SPECIFICATION_FILES/Ey.tout_ref",
    **{f"tem_{a.lower()}_aniso_{p.lower()}": f"TEM_{a}_ANISOTROPIC_THIN_LAYER_{p}_POL_TEST/PROBLEM_SPECIFICATION_FILES/Ey.tout_ref"
       for a, p in (("X", "Y"), ("X", "Z"), ("Y", "X"), ("Y", "Z"), ("Z", "X"), ("Z", "Y"))},
    "thin_layer_stability": "THIN_LAYER_STABILITY_TEST/PROBLEM_SPECIFICATION_FILES/cavity.field.tout_ref",
    "wrapping_Ex": "WRAPPING_BOUNDARY/PROBLEM_SPECIFICATION_FILES/Ex_centre.tout_ref",
    # Debye and eps_r = 1.5 blocks with PEC and dispersive thin-layer sheets
    "material_test_Ex": "MATERIAL_TEST/PROBLEM_SPECIFICATION_FILES/mat_test.field.tout_ref",
    # volume average 1 of a wrapped cell with an FR4 slab, PEC patches and a Huygens plane
    # (post-processor option 1 on the run's .volume_average_field.tout); first 20000 of 59958 steps kept
    "resonant_absorber_Ey": "RESONANT_ABSORBER/PROBLEM_SPECIFICATION_FILES/Ey.tout_ref",
}
# cases whose golden series is cut to its first rows
CASE_ROWS = {"resonant_absorber_Ey": 20000}


# raw text of the reference's .tout files (header and every data line), kept
# to check that the library's .tout writer reproduces them byte for byte
TEXT_CASES = ["tem_pml_Ey", "material_test2_Ex", "huygens_box_Hz"]
VMAT_CASES = ["debye_1", "debye_2", "FR4_at_7GHz", "mur_lorentz", "epsr=2", "mur=2", "epsr=1.5"]
# the known-answer cases' problem input files, as text, for the .inp reader;
# read as Latin-1 since their remarks hold stray non-ASCII bytes
INP_CASES = {
    "tem_pml": "TEM_PML_TEST/PROBLEM_SPECIFICATION_FILES/TEM_cell.inp",
    "tem_material": "TEM_MATERIAL_TEST/PROBLEM_SPECIFICATION_FILES/TEM_cell.inp",
    "material_stability": "MATERIAL_STABILITY_TEST/PROBLEM_SPECIFICATION_FILES/cavity.inp",
    "material_test2": "MATERIAL_TEST2/PROBLEM_SPECIFICATION_FILES/mat_test.inp",
    "huygens_box": "HUYGENS_SURFACE/PROBLEM_SPECIFICATION_FILES/huygens_test.inp",
    "cavity_free_space": "CAVITY_FREE_SPACE/PROBLEM_SPECIFICATION_FILES/cavity_1_2_3.inp",
    "cavity_epsr2": "CAVITY_EPSR=2/PROBLEM_SPECIFICATION_FILES/cavity_1_2_3.inp",
    "cavity_mur2": "CAVITY_MUR=2/PROBLEM_SPECIFICATION_FILES/cavity_1_2_3.inp",
    "parallel_test": "PARALLEL_TEST/PROBLEM_SPECIFICATION_FILES/cavity.inp",
    "box_slot": "SHIELDING_EFFECTIVENESS_BOX_SLOT/PROBLEM_SPECIFICATION_FILES/box_slot.inp",
    "excitation_test": "EXCITATION_FUNCTION_TEST/PROBLEM_SPECIFICATION_FILES/excitation_test.inp",
    "power_calc": "POWER_CALCS/PROBLEM_SPECIFICATION_FILES/power_calc.inp",
    "helix": "HELIX_ANTENNA/helix.inp",
    "rcs_plate": "RCS_PEC_PLATE_ROUGH_SURFACE/PROBLEM_SPECIFICATION_FILES/plate.inp",
    "tem_thin_layer": "TEM_THIN_LAYER_TEST/PROBLEM_SPECIFICATION_FILES/TEM_cell.inp",
    **{f"tem_{a.lower()}_aniso_{p.lower()}": f"TEM_{a}_ANISOTROPIC_THIN_LAYER_{p}_POL_TEST/PROBLEM_SPECIFICATION_FILES/TEM_cell.inp"
       for a, p in (("X", "Y"), ("X", "Z"), ("Y", "X"), ("Y", "Z"), ("Z", "X"), ("Z", "Y"))},
    "thin_layer_stability": "THIN_LAYER_STABILITY_TEST/PROBLEM_SPECIFICATION_FILES/cavity.inp",
    "wrapping": "WRAPPING_BOUNDARY/PROBLEM_SPECIFICATION_FILES/wrapping_test.inp",
    # a frequency selective surface: two square PEC loops in a cell wrapped in x and y, a normally
    # incident plane wave (the case's parameter set 4, which its S21.fout_4_ref is from)
    "fss_single_cell": "PARAMETERISED_FSS/PROBLEM_SPECIFICATION_FILES/single_cell.inp",
    "material_test": "MATERIAL_TEST/PROBLEM_SPECIFICATION_FILES/mat_test.inp",
    "resonant_absorber": "RESONANT_ABSORBER/PROBLEM_SPECIFICATION_FILES/TEM_cell.inp",
    # a PEC waveguide cavity driven by a soft Ex excitation surface across its cross section
    "waveguide": "WAVEGUIDE_RESONATOR/PROBLEM_SPECIFICATION_FILES/waveguide.inp",
    # WR90 waveguides driven by a TE10 mode excitation from a mode file, ended by mode-impedance
    # thin layers: straight, with a PML, and with an iris
    "waveguide_straight": "WAVEGUIDE_STRAIGHT/PROBLEM_SPECIFICATION_FILES/waveguide_straight.inp",
    "waveguide_pml": "WAVEGUIDE_PML/PROBLEM_SPECIFICATION_FILES/waveguide_pml.inp",
    "waveguide_iris": "WAVEGUIDE_IRIS/PROBLEM_SPECIFICATION_FILES/waveguide_iris.inp",
}
# the surface material files the thin-layer cases use, as text
SMAT_CASES = ["Dispersive_sheet", "Anisotropic_sheet", "WR90_mode_impedance"]
# result files the solver writes after the run (write_SAR_volumes), as text
RESULT_CASES = {
    "sar_test": "SAR_TEST/PROBLEM_SPECIFICATION_FILES/SAR_test.SAR.fout_ref",
    "rcs_plate_fout": "RCS_PEC_PLATE_ROUGH_SURFACE/PROBLEM_SPECIFICATION_FILES/plate.rcs.fout_ref",
    "rcs_plate_tout": "RCS_PEC_PLATE_ROUGH_SURFACE/PROBLEM_SPECIFICATION_FILES/plate.rcs.tout_ref",
}
# the head of long result files: (file, number of leading lines kept)
RESULT_HEADS = {
    # HELIX_ANTENNA's surface field file: the template of its one output
    # surface and the first data frame (output_surfaces.F90:326-927)
    "helix_surface_field": ("HELIX_ANTENNA/helix.surface_field.tout", 10603),
    # the mode-excited waveguides' time-domain results, whole
    "waveguide_straight_mode": ("WAVEGUIDE_STRAIGHT/PROBLEM_SPECIFICATION_FILES/waveguide_straight.mode.tout_ref", None),
    "waveguide_straight_field": ("WAVEGUIDE_STRAIGHT/PROBLEM_SPECIFICATION_FILES/waveguide_straight.field.tout_ref",
                                 None),
    "waveguide_pml_Ex1": ("WAVEGUIDE_PML/PROBLEM_SPECIFICATION_FILES/Ex1.tout_ref", None),
    "waveguide_iris_field": ("WAVEGUIDE_IRIS/PROBLEM_SPECIFICATION_FILES/waveguide_iris.field.tout_ref", None),
}
# mesh files written by the reference's mesher (MESH/write_mesh.F90), as text
MESH_CASES = {
    "helix": "HELIX_ANTENNA/helix.mesh",
}
# the post-processor's input files of the cases whose post-processed results are golden, as text
POST_CASES = {
    "power_calc": "POWER_CALCS/PROBLEM_SPECIFICATION_FILES/GGI_TLM_post_process_in.txt",
    "fss": "PARAMETERISED_FSS/PROBLEM_SPECIFICATION_FILES/GGI_TLM_post_process_in.txt",
    "resonant_absorber": "RESONANT_ABSORBER/PROBLEM_SPECIFICATION_FILES/GGI_TLM_post_process_in.txt",
    "box_slot": "SHIELDING_EFFECTIVENESS_BOX_SLOT/PROBLEM_SPECIFICATION_FILES/GGI_TLM_post_process_in.txt",
    "waveguide": "WAVEGUIDE_RESONATOR/PROBLEM_SPECIFICATION_FILES/GGI_TLM_post_process_in.txt",
    "waveguide_straight": "WAVEGUIDE_STRAIGHT/PROBLEM_SPECIFICATION_FILES/GGI_TLM_post_process_in.txt",
    "waveguide_pml": "WAVEGUIDE_PML/PROBLEM_SPECIFICATION_FILES/GGI_TLM_post_process_in.txt",
    "waveguide_iris": "WAVEGUIDE_IRIS/PROBLEM_SPECIFICATION_FILES/GGI_TLM_post_process_in.txt",
}
# data files the inputs name (excitation function samples), as text
DATA_CASES = {
    "gaussian_from_file.dat": "EXCITATION_FUNCTION_TEST/PROBLEM_SPECIFICATION_FILES/gaussian_from_file.dat",
    # each waveguide case's own mode file (NAME@case)
    "WR90.mode@waveguide_straight": "WAVEGUIDE_STRAIGHT/PROBLEM_SPECIFICATION_FILES/WR90.mode",
    "WR90.mode@waveguide_pml": "WAVEGUIDE_PML/PROBLEM_SPECIFICATION_FILES/WR90.mode",
    "WR90.mode@waveguide_iris": "WAVEGUIDE_IRIS/PROBLEM_SPECIFICATION_FILES/WR90.mode",
}
# the post-processor's Fourier transforms of those four cases' output point
# (GGI_TLM_post_process_in.txt beside each: option 3, point 1, lin 1 MHz to
# 300 MHz, 1000 frequencies; 100 for PARALLEL_TEST), as text
FOUT_CASES = {
    "cavity_free_space": "CAVITY_FREE_SPACE/PROBLEM_SPECIFICATION_FILES/cavity_1_2_3.fout_ref",
    "cavity_epsr2": "CAVITY_EPSR=2/PROBLEM_SPECIFICATION_FILES/cavity_1_2_3.fout_ref",
    "cavity_mur2": "CAVITY_MUR=2/PROBLEM_SPECIFICATION_FILES/cavity_1_2_3.fout_ref",
    "parallel_test": "PARALLEL_TEST/PROBLEM_SPECIFICATION_FILES/cavity.fout_ref",
    # option 3 on the excitation and on the probe, then option 6: excitation / probe
    "box_slot": "SHIELDING_EFFECTIVENESS_BOX_SLOT/PROBLEM_SPECIFICATION_FILES/Shielding_effectiveness.fout_ref",
    # written by the solver itself (write_frequency_domain_power_surfaces)
    "power_calc": "POWER_CALCS/PROBLEM_SPECIFICATION_FILES/power_calc.frequency_domain_power_surface.fout_ref",
    # four volume averages Fourier transformed (option 3), then the one-port analysis (option 9)
    "resonant_absorber": "RESONANT_ABSORBER/PROBLEM_SPECIFICATION_FILES/Resonant_absorber.fout_ref",
    # option 15, transmission cross section, from the power surface file and the field spectrum
    "power_calc_tcs": "POWER_CALCS/PROBLEM_SPECIFICATION_FILES/TCS.fout_ref",
    # eight volume averages Fourier transformed (option 3), then the two-port analysis (option 10)
    "fss_s21": "PARAMETERISED_FSS/PROBLEM_SPECIFICATION_FILES/S21.fout_4_ref",
    # option 3 on output point 1 (8 GHz to 12 GHz, 800 frequencies), then option 13: the mode on
    # the frequency output surface
    "waveguide": "WAVEGUIDE_RESONATOR/PROBLEM_SPECIFICATION_FILES/waveguide.field.fout_ref",
    "waveguide_mode": "WAVEGUIDE_RESONATOR/PROBLEM_SPECIFICATION_FILES/WR90.mode_ref",
    # the mode-excited waveguides: four mode outputs Fourier transformed (option 3), then the one-port
    # (option 9) or, for the iris, eight, then the two-port analysis (option 10)
    "waveguide_straight": "WAVEGUIDE_STRAIGHT/PROBLEM_SPECIFICATION_FILES/waveguide_straight.fout_ref",
    "waveguide_pml": "WAVEGUIDE_PML/PROBLEM_SPECIFICATION_FILES/waveguide_pml.fout_ref",
    "waveguide_iris": "WAVEGUIDE_IRIS/PROBLEM_SPECIFICATION_FILES/waveguide_iris.fout_ref",
}


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GGI_TLM_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py <reference checkout> (or set GGI_TLM_REFERENCE)")
    here = os.path.dirname(os.path.abspath(__file__))
    for name, rel in CASES.items():
        path = os.path.join(ref, "GGI_TLM", "TEST_DATA", rel)
        d = np.loadtxt(path, comments="#")[:CASE_ROWS.get(name)]
        np.savez_compressed(os.path.join(here, name + ".npz"), time=d[:, 0], point=d[:, 1].astype(np.int32),
                            value=d[:, 2], source=rel)
        print(name, d.shape)
    lines = {}
    for name in TEXT_CASES:
        with open(os.path.join(ref, "GGI_TLM", "TEST_DATA", CASES[name])) as f:
            lines[name] = np.array(f.read().splitlines())
    np.savez_compressed(os.path.join(here, "tout_text.npz"), **lines)
    print("tout_text", {k: len(v) for k, v in lines.items()})
    # the reference's volume material files that its known-answer cases use, as text
    vm = {}
    for name in VMAT_CASES:
        with open(os.path.join(ref, "GGI_TLM", "TEST_DATA", "MATERIAL_DATA", name + ".vmat")) as f:
            vm[name] = np.array(f.read().splitlines())
    np.savez_compressed(os.path.join(here, "vmat_text.npz"), **vm)
    print("vmat_text", sorted(vm))
    sm = {}
    for name in SMAT_CASES:
        with open(os.path.join(ref, "GGI_TLM", "TEST_DATA", "MATERIAL_DATA", name + ".smat")) as f:
            sm[name] = np.array(f.read().splitlines())
    np.savez_compressed(os.path.join(here, "smat_text.npz"), **sm)
    print("smat_text", sorted(sm))
    inp = {}
    for name, rel in INP_CASES.items():
        with open(os.path.join(ref, "GGI_TLM", "TEST_DATA", rel), encoding="latin-1") as f:
            inp[name] = np.array(f.read().splitlines())
    np.savez_compressed(os.path.join(here, "inp_text.npz"), **inp)
    print("inp_text", {k: len(v) for k, v in inp.items()})
    pp = {}
    for name, rel in POST_CASES.items():
        with open(os.path.join(ref, "GGI_TLM", "TEST_DATA", rel), encoding="latin-1") as f:
            pp[name] = np.array(f.read().splitlines())
    np.savez_compressed(os.path.join(here, "post_process_text.npz"), **pp)
    print("post_process_text", {k: len(v) for k, v in pp.items()})
    data = {}
    for name, rel in DATA_CASES.items():
        with open(os.path.join(ref, "GGI_TLM", "TEST_DATA", rel), encoding="latin-1") as f:
            data[name] = np.array(f.read().splitlines())
    np.savez_compressed(os.path.join(here, "data_text.npz"), **data)
    print("data_text", {k: len(v) for k, v in data.items()})
    fo = {}
    for name, rel in FOUT_CASES.items():
        with open(os.path.join(ref, "GGI_TLM", "TEST_DATA", rel)) as f:
            fo[name] = np.array(f.read().splitlines())
    np.savez_compressed(os.path.join(here, "fout_text.npz"), **fo)
    print("fout_text", {k: len(v) for k, v in fo.items()})
    rs = {}
    for name, rel in RESULT_CASES.items():
        with open(os.path.join(ref, "GGI_TLM", "TEST_DATA", rel)) as f:
            rs[name] = np.array(f.read().splitlines())
    for name, (rel, n_lines) in RESULT_HEADS.items():
        with open(os.path.join(ref, "GGI_TLM", "TEST_DATA", rel)) as f:
            rs[name] = np.array(f.read().splitlines()[:n_lines])  # None: every line
    np.savez_compressed(os.path.join(here, "result_text.npz"), **rs)
    print("result_text", {k: len(v) for k, v in rs.items()})
    me = {}
    for name, rel in MESH_CASES.items():
        with open(os.path.join(ref, "GGI_TLM", "TEST_DATA", rel)) as f:
            me[name] = np.array(f.read().splitlines())
    np.savez_compressed(os.path.join(here, "mesh_text.npz"), **me)
    print("mesh_text", {k: len(v) for k, v in me.items()})


if __name__ == "__main__":
    main()
