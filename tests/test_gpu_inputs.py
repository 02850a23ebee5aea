"""system.load_inputs with the harmonic stage on the device (fp4_eigen_dm)
gives the same solve as with the numpy restatement, up to the eigensolver's
freedom inside degenerate sets."""
import pytest

import harmonic_cases as HC
import helpers  # noqa: F401  (puts the repository on the path)
from fourphonon_b200 import crystal as C
from fourphonon_b200 import ifcgen as G
from fourphonon_b200 import inputs as I
from fourphonon_b200 import system as S

pytestmark = pytest.mark.gpu


def test_load_inputs_device_harmonic(tmp_path):
    from fourphonon_b200 import abi
    cr = C.diamond(5.43, (28.085, 28.085))
    cr.scell = (3, 3, 3)
    blocks = G.bvk_fc2(cr, [3.0, 0.45])
    shells = G.shell_distances(cr, 4)
    cl3 = G.generate_anharmonic(cr, 3, 0.5 * (shells[2] + shells[3]), 5.0, 11)
    I.write_control(tmp_path / "CONTROL", cr, (6, 6, 6), T=300.0, four_phonon=False)
    G.write_fc2_phonopy(tmp_path / "FORCE_CONSTANTS_2ND", cr, blocks)
    G.write_fc_anharmonic(tmp_path / "FORCE_CONSTANTS_3RD", cr, cl3)
    ctx = abi.Context(0)
    try:
        dev = S.load_inputs(str(tmp_path), ctx=ctx)
    finally:
        ctx.close()
    host = S.load_inputs(str(tmp_path))
    assert dev.ifc4 is None and dev.ifc3.ntri == host.ifc3.ntri
    HC.compare_harmonic((dev.energy, dev.velocity, dev.eig), (host.energy, host.velocity, host.eig),
                        omega_rtol=1e-11, vec_tol=1e-7, vel_rtol=1e-8)
