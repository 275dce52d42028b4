"""ctypes binding of libpfem2gpu.so (the C ABI declared in include/pfem2gpu.h).

There is no CPU fallback: if the library is missing or no CUDA device is
present, the calls fail with an exception.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
# PFEM2GPU_LIB selects another build of the same library (for comparing two
# builds in one process environment); by default the in-tree build.
LIB_PATH = os.environ.get("PFEM2GPU_LIB") or os.path.join(HERE, "_build", "libpfem2gpu.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "pfem2gpu.h")

OK = 0
FP64 = 0
FP32 = 1
ERRORS = {
    1: "invalid argument",
    2: "CUDA error",
    3: "call out of order",
    4: "particle capacity exceeded",
    5: "device out of memory",
    6: "no CUDA device",
    7: "kernel reported invalid data",
    8: "mesh larger than the static scratch of pfem2gpu_project_noalloc",
}
ERR_ARG = 1
ERR_CUDA = 2
ERR_STATE = 3
ERR_CAPACITY = 4
ERR_NOMEM = 5
ERR_NODEVICE = 6
ERR_DEVICE = 7
ERR_SCRATCH = 8


class Pfem2GpuError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__(f"pfem2gpu error {code} ({ERRORS.get(code, 'unknown')}){': ' + msg if msg else ''}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("particles_per_cell", C.c_int32 * 3),
        ("max_particles_per_cell_part", C.c_int32),
        ("particle_integration_steps", C.c_int32),
        ("time_step", C.c_double),
        ("removal_seed", C.c_uint32),
        ("empty_dof_policy", C.c_int32),
        ("capacity", C.c_int64),
        ("integrator", C.c_int32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("n_particles", C.c_int64),
        ("lost", C.c_int64),
        ("removed", C.c_int64),
        ("seeded", C.c_int64),
        ("map_failures", C.c_int64),
        ("near_face", C.c_int64),
        ("searched", C.c_int64),
        ("nan_dofs", C.c_int64),
        ("fallback64", C.c_int64),
        ("particle_steps", C.c_int64),
        ("next_id", C.c_uint32),
        ("error_flags", C.c_uint32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def declared_symbols():
    """Function names declared in include/pfem2gpu.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(pfem2gpu_[a-z_0-9]+)\s*\(", text)))


_lib = None


def load():
    """Load the shared library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} missing: build it with `python -m pfem2dealii_b200.build`")
    L = C.CDLL(LIB_PATH)
    P, i64, u32, dptr = C.c_void_p, C.c_int64, C.c_uint32, C.c_void_p
    sig = {
        "pfem2gpu_create": [C.c_int, C.c_int, C.POINTER(Params), C.POINTER(P)],
        "pfem2gpu_destroy": [P],
        "pfem2gpu_set_mesh": [P, i64, i64, i64, dptr, dptr, dptr, dptr, dptr, dptr],
        "pfem2gpu_seed": [P, dptr],
        "pfem2gpu_correct": [P, dptr, dptr],
        "pfem2gpu_move": [P, dptr],
        "pfem2gpu_project": [P, dptr],
        "pfem2gpu_seed_device": [P, dptr],
        "pfem2gpu_correct_device": [P, dptr, dptr],
        "pfem2gpu_move_device": [P, dptr],
        "pfem2gpu_project_device": [P, dptr],
        "pfem2gpu_step_device": [P, dptr, dptr, dptr],
        "pfem2gpu_correct_from_projection": [P, dptr],
        "pfem2gpu_correct_from_projection_device": [P, dptr],
        "pfem2gpu_get_particles": [P, dptr, dptr, dptr, dptr, dptr, i64, C.POINTER(i64)],
        "pfem2gpu_set_particles": [P, i64, dptr, dptr, dptr, dptr, dptr, u32],
        "pfem2gpu_set_partition": [P, i64, i64],
        "pfem2gpu_move_exchange_begin": [P, dptr, C.POINTER(i64)],
        "pfem2gpu_move_outbox": [P, dptr, dptr, dptr, dptr, dptr, i64, C.POINTER(i64)],
        "pfem2gpu_move_inbox": [P, i64, dptr, dptr, dptr, dptr, dptr, C.POINTER(i64)],
        "pfem2gpu_move_exchange_end": [P, u32, u32],
        "pfem2gpu_get_partials": [P, i64, dptr, dptr],
        "pfem2gpu_set_partials": [P, i64, dptr, dptr],
        "pfem2gpu_write_vtu": [P, C.c_char_p],
        "pfem2gpu_pack_output_device": [P, dptr, i64, C.POINTER(i64)],
        "pfem2gpu_get_stats": [P, C.POINTER(Stats)],
        "pfem2gpu_reset_stats": [P],
        "pfem2gpu_synchronize": [P],
        "pfem2gpu_get_stream": [P, C.POINTER(P)],
        "pfem2gpu_host_register": [P, C.c_size_t],
        "pfem2gpu_host_unregister": [P],
        "pfem2gpu_profile": [P, C.c_int],
        "pfem2gpu_profile_report": [P, C.c_char_p, i64],
        "pfem2gpu_launch_count": [P, C.POINTER(C.c_uint64)],
        "pfem2gpu_last_error": [P, C.c_char_p, i64],
        "pfem2gpu_window_forward_device": [P, C.c_int32, C.c_int32, dptr, dptr, dptr, dptr],
        "pfem2gpu_window_backward_device": [P, dptr, dptr, dptr, dptr],
        "pfem2gpu_adjoint": [P, C.c_int32, C.c_int32, dptr, dptr, dptr, dptr, dptr, dptr, dptr, dptr],
        "pfem2gpu_window_size": [P, C.POINTER(i64)],
        "pfem2gpu_window_particles": [P, dptr, dptr, dptr, i64, C.POINTER(i64)],
        "pfem2gpu_get_vertex_maps": [P, dptr, dptr, dptr, i64, C.POINTER(i64)],
        "pfem2gpu_fem_pattern": [P, dptr, dptr, i64, C.POINTER(i64)],
        "pfem2gpu_fem_set_boundary": [P, dptr, C.c_int32, dptr, C.c_int32, dptr],
        "pfem2gpu_fem_constrain": [P, C.c_int, C.c_int32, dptr, dptr, dptr, dptr],
        "pfem2gpu_fem_velocity_bc": [P, C.c_double, C.c_double, dptr, C.c_int32, dptr, dptr, dptr, dptr, i64,
                                     C.POINTER(i64)],
        "pfem2gpu_fem_constrain_device": [P, C.c_int, C.c_int32, dptr, dptr, dptr, dptr],
        "pfem2gpu_fem_assemble_device": [P, C.c_int, C.c_double, C.c_double, C.c_double, dptr, dptr, dptr, dptr,
                                         dptr],
        "pfem2gpu_fem_assemble": [P, C.c_int, C.c_double, C.c_double, C.c_double, dptr, dptr, dptr, dptr, dptr],
        "pfem2gpu_read_unv": [C.c_char_p, C.c_int, C.POINTER(C.c_int32), C.POINTER(i64), C.POINTER(i64), dptr, dptr,
                              i64, i64],
        "pfem2gpu_read_unv_error": [],
        "pfem2gpu_project_noalloc": [C.c_int, C.c_int32, C.c_int32, dptr, i64, dptr, dptr, dptr, C.c_int, dptr,
                                     C.POINTER(i64), P],
    }
    for name, argt in sig.items():
        f = getattr(L, name)
        f.argtypes = argt
        f.restype = C.c_int
    L.pfem2gpu_error_string.argtypes = [C.c_int]
    L.pfem2gpu_error_string.restype = C.c_char_p
    L.pfem2gpu_read_unv_error.restype = C.c_char_p
    _lib = L
    return L


def check(rc, h=None):
    if rc != OK:
        msg = ""
        if h:
            buf = C.create_string_buffer(1024)
            load().pfem2gpu_last_error(h, buf, 1024)
            msg = buf.value.decode(errors="replace")
        raise Pfem2GpuError(rc, msg)
