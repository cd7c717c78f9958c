"""The drop-in executable end to end on the GPU: gpu-vah reads the reference's
.properties files, runs the hydro loop and writes the reference's .dat files
(through the asynchronous writer), including the validity files when
VAH_VALIDITY=1. The CPU oracle, started from the executable's own first
output, reproduces its later outputs."""
import os
import subprocess

import numpy as np
import pytest

import vahlib as V

pytestmark = pytest.mark.gpu
EXE = os.path.join(V.ROOT, "gpu-vah_b200", "gpu-vah")
NX, NY, T0, DT = 21, 19, 0.5, 0.02


def write_config(d):
    with open(os.path.join(d, "lattice.properties"), "w") as f:
        f.write(f"numLatticePointsX = {NX}\nnumLatticePointsY = {NY}\nnumLatticePointsRapidity = 1\n"
                "numProperTimePoints = 20\nlatticeSpacingX = 0.2\nlatticeSpacingY = 0.2\n"
                f"latticeSpacingRapidity = 0.2\nlatticeSpacingProperTime = {DT}\n")
    with open(os.path.join(d, "ic.properties"), "w") as f:
        f.write("initialConditionType = 2\nnumberOfNucleonsPerNuclei = 197\nscatteringCrossSectionNN = 42.0\n"
                "impactParameter = 7.0\nfractionOfBinaryCollisions = 0.15\n")
    with open(os.path.join(d, "hydro.properties"), "w") as f:
        f.write(f"initialProperTimePoint = {T0}\nshearViscosityToEntropyDensity = 0.2\n"
                "freezeoutTemperatureGeV = 0.155\ninitializePimunuNavierStokes = 0\n")


def dat(d, name, t):
    a = np.loadtxt(os.path.join(d, f"{name}_{t:.3f}.dat"))
    assert a.shape == (NX * NY, 4)
    return a[:, 3]


def close(a, b, rel=1e-8, absolute=2e-8):
    """Printed values (%.8f) against the oracle's."""
    return np.max(np.abs(a - b)) <= absolute + rel * np.max(np.abs(b))


def test_gpu_vah_executable_matches_oracle(tmp_path):
    cfg, out = tmp_path / "conf", tmp_path / "out"
    cfg.mkdir()
    out.mkdir()
    write_config(str(cfg))
    env = dict(os.environ, VAH_PHYSICS="pimunu", VAH_EOS="conformal", VAH_VALIDITY="1")
    run = subprocess.run([EXE, "-c", str(cfg), "-o", str(out), "-h"], capture_output=True, text=True, env=env,
                         timeout=300)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr[-2000:]
    assert "Average time/step" in run.stdout

    g = V.Grid(NX, NY, 1, 0.2, 0.2, 0.2, 0.2, physics="pimunu", eos="conformal")
    e0 = dat(str(out), "e", T0)
    full = np.zeros(g.shape)
    full[2:-2, 2:-2, 2:-2] = e0.reshape(1, NY, NX)
    o = V.Oracle(g)
    V.load_state(o, {V.E: full.ravel(), V.PP: full.ravel() / 3, V.UT: np.ones(g.ncell)})
    o.set_conserved(T0, 0)  # the reference's initial P_L = 0.0154483 e, as the executable sets it
    o.set_ghost_cells()
    o.set_validity(1)
    t = T0
    for block in range(2):
        o.run(t, DT, 10)
        t = T0 + 10 * (block + 1) * DT
        for fid, name in ((V.E, "e"), (V.PL, "pl"), (V.UT, "ut"), (V.UX, "ux"), (V.UY, "uy"), (V.PITT, "pitt"),
                          (V.PIXX, "pixx")):
            assert close(dat(str(out), name, t), g.interior(o.field(fid)).ravel()), (name, t)
        for vid in (0, 2, 4, 6, 16):  # Knudsen numbers, Rpi, Rpi2, the regulator's factor
            name = V.product.VALIDITY_NAMES[vid]
            assert close(dat(str(out), name, t), g.interior(o.validity(vid)).ravel(), rel=1e-6), (name, t)


def test_gpu_vah_executable_runs_the_fp32_form(tmp_path):
    """VAH_PRECISION=fp32 runs the same program in the FP32 form: its outputs
    track the oracle's FP64 evolution within 1e-4 (normwise) after 20 steps."""
    cfg, out = tmp_path / "conf", tmp_path / "out"
    cfg.mkdir()
    out.mkdir()
    write_config(str(cfg))
    env = dict(os.environ, VAH_PHYSICS="pimunu", VAH_EOS="conformal", VAH_PRECISION="fp32")
    run = subprocess.run([EXE, "-c", str(cfg), "-o", str(out), "-h"], capture_output=True, text=True, env=env,
                         timeout=300)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr[-2000:]
    g = V.Grid(NX, NY, 1, 0.2, 0.2, 0.2, 0.2, physics="pimunu", eos="conformal")
    e0 = dat(str(out), "e", T0)
    full = np.zeros(g.shape)
    full[2:-2, 2:-2, 2:-2] = e0.reshape(1, NY, NX)
    o = V.Oracle(g)
    V.load_state(o, {V.E: full.ravel(), V.PP: full.ravel() / 3, V.UT: np.ones(g.ncell)})
    o.set_conserved(T0, 0)
    o.set_ghost_cells()
    o.run(T0, DT, 20)
    t = T0 + 20 * DT
    for fid, name in ((V.E, "e"), (V.PL, "pl"), (V.UT, "ut"), (V.UX, "ux"), (V.UY, "uy")):
        assert close(dat(str(out), name, t), g.interior(o.field(fid)).ravel(), rel=1e-4, absolute=1e-7), name
