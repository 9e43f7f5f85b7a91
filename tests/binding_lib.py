"""ctypes front end of tests/binding/_build/libb200_binding.so (test
infrastructure): one system built by the reference's own code, run behind the
reference's SimulatorBase either by its MolecularDynamicsSimulator (CPU) or by
B200Simulator, the reference-side binding of this library's C ABI (GPU)."""
import ctypes as C
import os

import numpy as np

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "binding", "_build", "libb200_binding.so")
REFERENCE_MD, B200 = 0, 1


def available() -> bool:
    return os.path.exists(LIB)


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(LIB)
        _lib.bind_run.restype = C.c_int
        _lib.bind_run.argtypes = [C.POINTER(oracle.OrcSpec), C.c_int, C.c_int, C.c_longlong, C.c_char_p,
                                  C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _lib.bind_last_error.restype = C.c_char_p
    return _lib


def run(desc, where, steps, prefix, precision=0):
    """Velocity-Verlet run of `steps` steps (desc.dt); returns (pos, vel,
    total energy) after finalize()."""
    d = desc.copy()
    d.integrator = "VelocityVerlet"
    spec, keep = oracle.make_spec(d)
    pos, vel = np.empty((d.n, 3)), np.empty((d.n, 3))
    e = C.c_double(0.0)
    code = lib().bind_run(C.byref(spec), where, precision, steps, prefix.encode(),
                          pos.ctypes.data_as(C.POINTER(C.c_double)), vel.ctypes.data_as(C.POINTER(C.c_double)),
                          C.byref(e))
    if code != 0:
        raise RuntimeError(lib().bind_last_error().decode())
    del keep
    return pos, vel, e.value
