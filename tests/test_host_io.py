"""CF/SF text formats of the reference (src/hawaii.c:4150-4284) round-trip."""
import numpy as np

import hawaiihybrid_b200 as hh
from hawaiihybrid_b200 import hawaii as H


def test_cf_roundtrip(tmp_path):
    N = 64
    cf = hh.CFnc(t=np.linspace(0, 200.0 * (N - 1), N), data=np.exp(-np.arange(N) / 10.0) * 1e-33,
                 ntraj=1000.0, Temperature=300.0, normalized=False)
    cf.data *= cf.ntraj
    f = tmp_path / "cf.txt"
    hh.write_correlation_function(str(f), cf)
    lines = f.read_text().splitlines()
    assert lines[0] == "# HAWAII HYBRID v0.1"
    assert lines[1].startswith("# Saved on ")
    assert lines[2] == "# TEMPERATURE: 300.00"
    assert lines[3] == "# AVERAGE OVER 1000.00 TRAJECTORIES"
    assert lines[4] == "# MAXIMUM TRAJECTORY LENGTH: 64"
    assert lines[5] == f"0.00 {cf.data[0] / 1000.0:.10e}"
    back = hh.read_correlation_function(str(f))
    np.testing.assert_allclose(back.data, cf.data / cf.ntraj, rtol=1e-10)
    assert back.Temperature == 300.0 and back.ntraj == 1000.0 and back.normalized


def test_sf_roundtrip(tmp_path):
    N = 32
    sf = hh.SFnc(nu=np.arange(N) * 0.05, data=np.linspace(1, 2, N) * 1e-80, ntraj=5.0, Temperature=100.0,
                 normalized=True)
    f = tmp_path / "sf.txt"
    hh.write_spectral_function(str(f), sf)
    lines = f.read_text().splitlines()
    assert lines[4] == "# SPECTRAL FUNCTION LENGTH: 32"
    assert lines[5] == f"{0.0:.10f}   {1e-80:.10e}"
    back = hh.read_spectral_function(str(f))
    np.testing.assert_allclose(back.data, sf.data, rtol=1e-10)


def test_reads_reference_golden_header(tmp_path):
    f = tmp_path / "cf.txt"
    f.write_text("# HAWAII HYBRID v0.1\n# TEMPERATURE: 1000.00\n# AVERAGE OVER 500000000.00 TRAJECTORIES\n"
                 "# MAXIMUM TRAJECTORY LENGTH: 2\n0.00 9.0933032379e-33\n200.00 8.9179914869e-33\n")
    cf = hh.read_correlation_function(str(f))
    assert cf.ntraj == 5e8 and cf.Temperature == 1000.0 and cf.len == 2


def test_partition_function_and_params():
    ms = H.MoleculeSystem(H.SYSTEM_CO2_AR, 3.8e4, hh.LINEAR_MOLECULE, hh.ATOM, (2.8e5, 2.8e5, 0.0))
    assert ms.QP_SIZE == 10 and ms.Q_SIZE == 5
    pf = hh.analytic_full_partition_function_by_V(ms, 300.0)
    kT = 300.0 / H.HkT
    assert abs(pf / (4 * np.pi * (2 * np.pi * kT) ** 2.5 * 3.8e4 ** 1.5 * 2.8e5) - 1) < 1e-14
    c = hh.CalcParams(MaxTrajectoryLength=128).to_c()
    assert c.MaxTrajectoryLength == 128 and c.pair_state == 1


def test_rotor_linear_partition_function_matches_reference_log():
    """src/hawaii.c:5083-5085 for CH4-CO2; the reference's own run prints
    'Analytic partition function divided by V: 4.16497e+10' at 100 K
    (example_configs/CF-F-CH4-CO2-100.0.conf.out)."""
    from tests.helpers import II_CH4, II_CO2, MU_CH4CO2
    ms = H.MoleculeSystem(H.SYSTEM_CH4_CO2, MU_CH4CO2, hh.ROTOR, hh.LINEAR_MOLECULE, (II_CH4,) * 3,
                          (II_CO2, II_CO2, 0.0))
    assert ms.QP_SIZE == 16
    assert f"{hh.analytic_full_partition_function_by_V(ms, 100.0):.5e}" == "4.16497e+10"


def test_native_writers_match_the_reference_format(tmp_path):
    """hh_write_correlation_function_ext / hh_write_spectral_function_ext (the parallel
    formatter of the library, no device needed) write the reference's bytes: its header
    lines and one printf-formatted line per point, divided by ntraj unless normalized."""
    import numpy as np
    from hawaiihybrid_b200 import hawaii as H
    rng = np.random.default_rng(3)
    N = 10000
    cf = H.CFnc(t=200.0 * np.arange(N), data=rng.standard_normal(N) * 1e-60, ntraj=1234.0, Temperature=300.0,
                normalized=False)
    p = tmp_path / "cf.txt"
    n = H.write_correlation_function(str(p), cf)
    lines = p.read_text().splitlines()
    assert n == p.stat().st_size
    assert lines[0] == "# HAWAII HYBRID v0.1" and lines[1].startswith("# Saved on ")
    assert lines[2:5] == ["# TEMPERATURE: 300.00", "# AVERAGE OVER 1234.00 TRAJECTORIES",
                          f"# MAXIMUM TRAJECTORY LENGTH: {N}"]
    assert lines[5:] == ["%.2f %.10e" % (t, v / 1234.0) for t, v in zip(cf.t, cf.data)]
    back = H.read_correlation_function(str(p))
    np.testing.assert_allclose(back.data, cf.data / 1234.0, rtol=1e-10)
    sf = H.SFnc(nu=np.linspace(0, 500, N), data=rng.random(N), ntraj=10.0, Temperature=150.0, normalized=True)
    q = tmp_path / "sf.txt"
    H.write_spectral_function(str(q), sf)
    ls = q.read_text().splitlines()
    assert ls[4] == f"# SPECTRAL FUNCTION LENGTH: {N}"
    assert ls[5:] == ["%.10f   %.10e" % (a, b) for a, b in zip(sf.nu, sf.data)]
