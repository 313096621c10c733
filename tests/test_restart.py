"""Checkpoint and restart in OpenFOAM format (postProcess/cfdWriteOpenFoamField.m layout;
startFrom latestTime, initialize/cfdInitializeCase.m:57-58): fields written at full precision
and read back restart the steady loop bit for bit."""
import dataclasses

import numpy as np

from matlab_ufvm_b200 import case, polymesh


def test_field_round_trip(tmp_path):
    spec = case.cavity_case(6)
    m = spec.mesh
    rng = np.random.default_rng(3)
    R = m.n_cells + m.n_faces - m.n_interior
    U, p, md = rng.normal(size=(3, R)), rng.normal(size=R), rng.normal(size=m.n_faces)
    polymesh.write_time_directory(str(tmp_path), "7", spec, U, p, md)
    U0, p0, m0 = polymesh.read_time_directory(str(tmp_path), "7", m)
    assert np.array_equal(U0, U[:, :m.n_cells].T)
    assert np.array_equal(p0, p[:m.n_cells])
    walls = [pt for pt, t in zip(m.patches, spec.bc_p) if t != "empty"]
    assert np.array_equal(m0[:m.n_interior], md[:m.n_interior])
    for pt in walls:
        assert np.array_equal(m0[pt.start:pt.start + pt.n], md[pt.start:pt.start + pt.n])
    f = polymesh.read_field(str(tmp_path / "7" / "U"))
    assert f["class"] == "volVectorField" and set(f["boundary"]) == {pt.name for pt in m.patches}


def test_short_format_matches_reference_precision(tmp_path):
    spec = case.cavity_case(4)
    R = spec.mesh.n_cells + spec.mesh.n_faces - spec.mesh.n_interior
    polymesh.write_time_directory(str(tmp_path), "1", spec, np.full((3, R), 5.41752), np.full(R, -1.79671e-7),
                                  np.zeros(spec.mesh.n_faces), digits=5)
    txt = (tmp_path / "1" / "U").read_text()
    assert "(5.4175 5.4175 5.4175)" in txt
    assert "-1.7967e-07" in (tmp_path / "1" / "p").read_text()


def test_restart_continues_bit_exact(oracle_mod, tmp_path):
    spec = case.cavity_case(12, nu=0.01)
    straight = oracle_mod.OracleCase(spec)
    for _ in range(5):
        straight.iterate()
    first = oracle_mod.OracleCase(spec)
    for _ in range(3):
        first.iterate()
    polymesh.write_time_directory(str(tmp_path), "3", spec, first.get("U"), first.get("p"), first.get("mdot"))
    U0, p0, m0 = polymesh.read_time_directory(str(tmp_path), "3", spec.mesh)
    resumed = oracle_mod.OracleCase(dataclasses.replace(spec, U0=U0, p0=p0, mdot0=m0))
    for _ in range(2):
        resumed.iterate()
    for name in ("U", "p", "mdot"):
        assert np.array_equal(straight.get(name), resumed.get(name)), name
