"""The input files of the path: a synthetic cell written as CONTROL, a Phonopy
FORCE_CONSTANTS_2ND and FORCE_CONSTANTS_3RD/4TH, and read back by
system.load_inputs (the CONTROL reader, read2fc, read3fc/read4fc and the
numpy eigenDM), gives the same solve as the arrays it was written from."""
import numpy as np

import harmonic_cases as HC
import helpers  # noqa: F401  (puts the repository on the path)
from fourphonon_b200 import crystal as C
from fourphonon_b200 import harmonic as HM
from fourphonon_b200 import ifcgen as G
from fourphonon_b200 import inputs as I
from fourphonon_b200 import system as S


def test_written_inputs_load_back(tmp_path):
    cr = C.diamond(5.43, (28.085, 28.085))
    cr.scell = (3, 3, 3)
    ngrid = (4, 4, 4)
    blocks = G.bvk_fc2(cr, [3.0, 0.45])
    shells = G.shell_distances(cr, 4)
    cl3 = G.generate_anharmonic(cr, 3, 0.5 * (shells[2] + shells[3]), 5.0, 11)
    cl4 = G.generate_anharmonic(cr, 4, 0.5 * (shells[0] + shells[1]), 2.0, 12)
    I.write_control(tmp_path / "CONTROL", cr, ngrid, T=300.0, scalebroad=1.0, four_phonon=True)
    G.write_fc2_phonopy(tmp_path / "FORCE_CONSTANTS_2ND", cr, blocks)
    G.write_fc_anharmonic(tmp_path / "FORCE_CONSTANTS_3RD", cr, cl3)
    G.write_fc_anharmonic(tmp_path / "FORCE_CONSTANTS_4TH", cr, cl4)

    s = S.load_inputs(str(tmp_path))
    fc = S.fc2_array(cr, blocks)
    sym = C.build_symmetry(cr, ngrid)
    om, vel, eig = HM.eigen_dm(cr, fc, ngrid, sym.symmetrizers)
    assert s.ngrid == ngrid and s.temperatures == [300.0] and s.scalebroad == 1.0
    assert np.array_equal(s.wedge.list, C.wedge(sym).list)
    # eigenvectors and single velocities inside a degenerate set are the solver's choice
    HC.compare_harmonic((s.energy, s.velocity, s.eig), (om, vel, eig), omega_rtol=1e-11, vec_tol=1e-7,
                        vel_rtol=1e-8)
    for ifc, cl in ((s.ifc3, cl3), (s.ifc4, cl4)):
        ref = S.IFC.from_clusters(cl, cr.lattvec)
        assert ifc.ntri == ref.ntri
        assert np.array_equal(ifc.cells, ref.cells) and np.array_equal(ifc.atoms, ref.atoms)
        assert np.abs(ifc.phi - ref.phi).max() <= 1e-9


def test_control_without_masses_is_rejected(tmp_path):
    cr = C.diamond(5.43, (28.085, 28.085))
    I.write_control(tmp_path / "CONTROL", cr, (2, 2, 2), T=300.0)
    lines = (tmp_path / "CONTROL").read_text().splitlines()
    kept = [x for x in lines if not x.strip().startswith("masses=")]
    assert len(kept) == len(lines) - 1
    (tmp_path / "CONTROL").write_text("\n".join(kept) + "\n")
    try:
        S.load_inputs(str(tmp_path))
    except I.InputError:
        return
    raise AssertionError("a CONTROL without masses was accepted")


def _control_with(tmp_path, extra_params=(), flags=None):
    cr = C.diamond(5.43, (28.085, 28.085))
    I.write_control(tmp_path / "CONTROL", cr, (2, 2, 2), T=300.0, four_phonon=bool(flags and flags.get("four_phonon")))
    text = (tmp_path / "CONTROL").read_text()
    for line in extra_params:
        text = text.replace("&parameters\n", "&parameters\n        " + line + "\n", 1)
    if flags:
        for k, v in flags.items():
            val = ".TRUE." if v else ".FALSE."
            lines = [x for x in text.splitlines() if not x.strip().startswith(k + "=")]
            text = "\n".join(lines) + "\n"
            text = text.replace("&flags\n", f"&flags\n        {k}={val}\n", 1)
    (tmp_path / "CONTROL").write_text(text)
    return cr


def test_control_reads_phase_space_sampling_parameters(tmp_path):
    _control_with(tmp_path, ["num_sample_process_3ph_phase_space=1000", "num_sample_process_4ph_phase_space=2000"],
                  {"four_phonon": True})
    c = I.read_control(str(tmp_path / "CONTROL"))
    assert c.num_sample_process_3ph_phase_space == 1000
    assert c.num_sample_process_4ph_phase_space == 2000
    assert c.num_sample_process_3ph == -1 and c.num_sample_process_4ph == -1


def _rejected(path):
    try:
        I.read_control(path)
    except I.InputError:
        return True
    return False


def test_control_sampling_consistency_checks(tmp_path):
    # config.f90:204-221: 4ph sampling without four_phonon, 3ph sampling with convergence,
    # 4ph sampling with the 4ph iteration
    _control_with(tmp_path, ["num_sample_process_4ph_phase_space=10"], {"four_phonon": False})
    assert _rejected(str(tmp_path / "CONTROL"))
    _control_with(tmp_path, ["num_sample_process_3ph=10"], {"convergence": True})
    assert _rejected(str(tmp_path / "CONTROL"))
    _control_with(tmp_path, ["num_sample_process_4ph=10"],
                  {"four_phonon": True, "convergence": True, "four_phonon_iteration": True})
    assert _rejected(str(tmp_path / "CONTROL"))
    _control_with(tmp_path, ["num_sample_process_4ph=10"], {"four_phonon": True, "convergence": False})
    assert not _rejected(str(tmp_path / "CONTROL"))


def test_four_phonon_without_fc4_is_rejected(tmp_path):
    cr = C.diamond(5.43, (28.085, 28.085))
    cr.scell = (3, 3, 3)
    blocks = G.bvk_fc2(cr, [3.0, 0.45])
    shells = G.shell_distances(cr, 4)
    cl3 = G.generate_anharmonic(cr, 3, 0.5 * (shells[2] + shells[3]), 5.0, 11)
    I.write_control(tmp_path / "CONTROL", cr, (2, 2, 2), T=300.0, four_phonon=True)
    G.write_fc2_phonopy(tmp_path / "FORCE_CONSTANTS_2ND", cr, blocks)
    G.write_fc_anharmonic(tmp_path / "FORCE_CONSTANTS_3RD", cr, cl3)
    try:
        S.load_inputs(str(tmp_path))
    except I.InputError:
        return
    raise AssertionError("four_phonon=.TRUE. without FORCE_CONSTANTS_4TH was accepted")
