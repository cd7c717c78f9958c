"""The drop-in host surface (libvah_host.so, gpu-vah): .properties loading
with libconfig's typing and the reference defaults, the .dat writer's format,
and the command line. CPU only."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import vahlib as V

HOSTLIB = os.path.join(V.ROOT, "gpu-vah_b200", "libvah_host.so")
EXE = os.path.join(V.ROOT, "gpu-vah_b200", "gpu-vah")


class Lattice(C.Structure):
    _fields_ = [("numLatticePointsX", C.c_int), ("numLatticePointsY", C.c_int),
                ("numLatticePointsRapidity", C.c_int), ("numComputationalLatticePointsX", C.c_int),
                ("numComputationalLatticePointsY", C.c_int), ("numComputationalLatticePointsRapidity", C.c_int),
                ("numProperTimePoints", C.c_int), ("latticeSpacingX", C.c_double), ("latticeSpacingY", C.c_double),
                ("latticeSpacingRapidity", C.c_double), ("latticeSpacingProperTime", C.c_double)]


class IC(C.Structure):
    _fields_ = [("initialConditionType", C.c_int), ("numberOfNucleonsPerNuclei", C.c_int),
                ("initialEnergyDensity", C.c_double), ("scatteringCrossSectionNN", C.c_double),
                ("impactParameter", C.c_double), ("fractionOfBinaryCollisions", C.c_double),
                ("rapidityVariance", C.c_double), ("rapidityMean", C.c_double)]


class Hydro(C.Structure):
    _fields_ = [("initialProperTimePoint", C.c_double), ("shearViscosityToEntropyDensity", C.c_double),
                ("freezeoutTemperatureGeV", C.c_double), ("initializePimunuNavierStokes", C.c_int)]


@pytest.fixture(scope="module")
def host():
    V.make(os.path.join(V.ROOT, "gpu-vah_b200"), "libvah_host.so", "gpu-vah")
    L = C.CDLL(HOSTLIB)
    L.vah_load_lattice_parameters.argtypes = [C.c_char_p, C.POINTER(Lattice)]
    L.vah_load_initial_condition_parameters.argtypes = [C.c_char_p, C.POINTER(IC)]
    L.vah_load_hydro_parameters.argtypes = [C.c_char_p, C.POINTER(Hydro)]
    L.vah_output.argtypes = [C.POINTER(C.c_double), C.c_double, C.c_char_p, C.c_char_p, C.POINTER(Lattice)]
    return L


def write(d, name, text):
    with open(os.path.join(d, name), "w") as f:
        f.write(text)


def test_defaults_when_files_are_missing(host, tmp_path):
    lat, ic, hy = Lattice(), IC(), Hydro()
    assert host.vah_load_lattice_parameters(str(tmp_path).encode(), C.byref(lat)) == 1
    assert host.vah_load_initial_condition_parameters(str(tmp_path).encode(), C.byref(ic)) == 1
    assert host.vah_load_hydro_parameters(str(tmp_path).encode(), C.byref(hy)) == 1
    # LatticeParameters.cpp:30-39, InitialConditionParameters.cpp:33-41, HydroParameters.cpp:25-29
    assert (lat.numLatticePointsX, lat.numLatticePointsY, lat.numLatticePointsRapidity) == (128, 128, 64)
    assert lat.numProperTimePoints == 10 and lat.numComputationalLatticePointsX == 132
    assert (lat.latticeSpacingX, lat.latticeSpacingRapidity, lat.latticeSpacingProperTime) == (0.08, 0.3, 0.01)
    assert (ic.initialConditionType, ic.numberOfNucleonsPerNuclei) == (2, 208)
    assert (ic.initialEnergyDensity, ic.scatteringCrossSectionNN, ic.impactParameter) == (1.0, 62, 7)
    assert (ic.fractionOfBinaryCollisions, ic.rapidityVariance, ic.rapidityMean) == (0.5, 0.5, 0.5)
    assert (hy.initialProperTimePoint, hy.shearViscosityToEntropyDensity) == (0.1, 0.0795775)
    assert (hy.freezeoutTemperatureGeV, hy.initializePimunuNavierStokes) == (0.155, 1)


def test_values_and_libconfig_typing(host, tmp_path):
    write(tmp_path, "lattice.properties", "numLatticePointsX=201\nnumLatticePointsY = 3;\n"
                                          "numLatticePointsRapidity: 1 # comment\nnumProperTimePoints=10000\n"
                                          "latticeSpacingX=0.1\nlatticeSpacingY=1e-1\n"
                                          "latticeSpacingRapidity=1\n/* block */ latticeSpacingProperTime=0.005\n")
    write(tmp_path, "ic.properties", "# Initial condition\ninitialConditionType=4\nnumberOfNucleonsPerNuclei=197\n"
                                     "initialEnergyDensity=15.6269\nscatteringCrossSectionNN=42\n"
                                     "impactParameter=3.5\nfractionOfBinaryCollisions=1.0\n"
                                     "rapidityVariance=0.16\nrapidityMean=5.9\n")
    write(tmp_path, "hydro.properties", "initialProperTimePoint=0.25\nshearViscosityToEntropyDensity=0.2\n"
                                        "freezeoutTemperatureGeV=0.140\ninitializePimunuNavierStokes=0.0\n")
    lat, ic, hy = Lattice(), IC(), Hydro()
    d = str(tmp_path).encode()
    assert host.vah_load_lattice_parameters(d, C.byref(lat)) == 0
    assert host.vah_load_initial_condition_parameters(d, C.byref(ic)) == 0
    assert host.vah_load_hydro_parameters(d, C.byref(hy)) == 0
    assert (lat.numLatticePointsX, lat.numLatticePointsY, lat.numLatticePointsRapidity) == (201, 3, 1)
    assert lat.numProperTimePoints == 10000 and lat.latticeSpacingX == 0.1 and lat.latticeSpacingY == 0.1
    # an integer literal does not answer a float lookup: the default 0.3 stays
    assert lat.latticeSpacingRapidity == 0.3
    assert lat.latticeSpacingProperTime == 0.005
    assert (ic.initialConditionType, ic.numberOfNucleonsPerNuclei) == (4, 197)
    assert ic.scatteringCrossSectionNN == 62          # "42" is an integer literal -> default
    assert ic.impactParameter == 3.5 and ic.rapidityMean == 5.9
    assert hy.initialProperTimePoint == 0.25 and hy.freezeoutTemperatureGeV == 0.14
    assert hy.initializePimunuNavierStokes == 1       # "0.0" is a float literal -> default


def test_malformed_file_keeps_defaults(host, tmp_path, capfd):
    write(tmp_path, "hydro.properties", "initialProperTimePoint = = 3\n")
    hy = Hydro()
    assert host.vah_load_hydro_parameters(str(tmp_path).encode(), C.byref(hy)) == 1
    assert hy.initialProperTimePoint == 0.1
    assert "Using default hydrodynamic configuration parameters." in capfd.readouterr().err


def test_dat_writer_format(host, tmp_path):
    lat = Lattice(3, 2, 1, 7, 6, 5, 0, 0.2, 0.1, 0.3, 0.01)
    var = np.arange(7 * 6 * 5, dtype=np.float64) / 7.0
    assert host.vah_output(var.ctypes.data_as(V.P), 0.5, str(tmp_path).encode(), b"e", C.byref(lat)) == 0
    lines = open(os.path.join(tmp_path, "e_0.500.dat")).read().splitlines()
    assert len(lines) == 6
    # FileIO.cpp:46-56: eta outer, y, x inner over the interior
    expect = []
    for j in range(2, 4):
        for i in range(2, 5):
            s = i + 7 * (j + 6 * 2)
            expect.append("%.3f\t%.3f\t%.3f\t%.8f" % ((i - 2 - 1.0) * 0.2, (j - 2 - 0.5) * 0.1, 0.0, var[s]))
    assert lines == expect


def test_command_line_surface(host, tmp_path):
    out = subprocess.run([EXE, "--config", str(tmp_path), "-o", str(tmp_path)], capture_output=True, text=True)
    assert out.returncode == 0
    assert out.stdout.splitlines()[:4] == [f"configDirectory = {tmp_path}", f"outputDirectory = {tmp_path}",
                                          "runHydro = False", "runTest = False"]
    out = subprocess.run([EXE, "-c", str(tmp_path), "-t"], capture_output=True, text=True)
    assert "runTest = True" in out.stdout
