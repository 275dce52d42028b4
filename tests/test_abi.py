"""CPU checks of the C ABI library: it loads, exports every function the
header declares, rejects bad arguments, and reports a missing device with
an error code instead of crashing."""
import ctypes as C
import os
import subprocess

import pytest

from pfem2dealii_b200 import _lib, build
from pfem2dealii_b200.handler import ParticleParams, read_prm


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def test_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    declared = _lib.declared_symbols()
    assert len(declared) >= 25
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    for s in declared:
        assert hasattr(lib, s)


def test_library_is_built_for_sm100a():
    log = open(build.os.path.join(build.OUT, "build.log")).read()
    assert "arch=compute_100a,code=sm_100a" in log
    assert "--fmad=false" in log  # FP64 form


def test_argument_validation(lib):
    h = C.c_void_p()
    p = ParticleParams(particles_per_cell=(2, 2, 2)).to_c(3)
    assert lib.pfem2gpu_create(4, 0, C.byref(p), C.byref(h)) == 1
    assert lib.pfem2gpu_create(3, 7, C.byref(p), C.byref(h)) == 1
    bad = ParticleParams(particles_per_cell=(0, 2, 2)).to_c(3)
    assert lib.pfem2gpu_create(3, 0, C.byref(bad), C.byref(h)) == 1
    big = ParticleParams(particles_per_cell=(9, 9, 9)).to_c(3)  # 1000 extended parts
    assert lib.pfem2gpu_create(3, 0, C.byref(big), C.byref(h)) == 1
    assert lib.pfem2gpu_destroy(None) == 1
    assert lib.pfem2gpu_error_string(4) == b"particle capacity exceeded"


def test_create_without_device_fails_cleanly(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    h = C.c_void_p()
    p = ParticleParams(particles_per_cell=(2, 2)).to_c(2)
    assert lib.pfem2gpu_create(2, 0, C.byref(p), C.byref(h)) == 6


def test_read_prm():
    text = """
subsection Computation parameters
    set Time step = 0.005
end
subsection Particles
    set Number of particles in the x direction = 3
    set Number of particles in the y direction = 2
    set Number of particles in the z direction = 4
    set Maximum number of particles per cell part = 5
    set Particle integration steps = 3
end
"""
    p = read_prm(text)
    assert p.particles_per_cell == (3, 2, 4)
    assert p.max_particles_per_cell_part == 5 and p.particle_integration_steps == 3 and p.time_step == 0.005


@pytest.mark.parametrize("case, q, maxpp, S, dt", [
    ("TurekBenchmark", (2, 2, 2), 5, 3, 0.001),
    ("PoiseuilleFlow3D", (2, 2, 2), 5, 3, 0.005),
    ("nacaAirfoil", (2, 2, 2), 5, 3, 0.001),
])
def test_read_prm_reference_cases(case, q, maxpp, S, dt):
    """The reference's own case files (cases/*/input_data.prm, committed as
    fixtures): the particle keys and the time step as its parameter handler
    reads them (src/pfem2parameterhandler.cpp:64-72,131-137); a missing z count is 2, its
    default, and a 2D handle uses the first two."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "prm", case + ".prm")
    p = read_prm(path)
    assert p.particles_per_cell == q
    assert p.max_particles_per_cell_part == maxpp and p.particle_integration_steps == S and p.time_step == dt

