"""NumPy-backed stand-in for ``cupy``, used only by tests/golden/make_golden.py.

It lets the reference's own Python orchestration (Grid, Boundary, CompTimes, T_OCEAN,
set_coords, set_weights, step2d, rhs3d, main3d) run unmodified on the CPU:

* array API: NumPy's, except that ``zeros``/``ones``/``empty``/``array`` return views into
  zero-guarded parent buffers, so that the reference kernels' out-of-bounds reads at the
  boundary ring (e.g. nonlinear/rhs_kernels.cpp:86-130 has no interior guard) read zeros
  instead of whatever memory precedes or follows an allocation;
* ``RawModule(code=...)`` recognises which reference kernel file it was given and binds
  ``get_function(name)`` to the host-compiled kernel in oracle/_ref (oracle/build_ref.py);
* a kernel call ``k(grid, block, args)`` runs grid*block threads in thread-index order and
  passes each argument as the kernel parameter type, using only as many arguments as the
  kernel declares.  That is what ``cuLaunchKernel`` does with CuPy's per-argument
  ``kernelParams`` array, and it is what makes the reference's mis-bound
  ``AdamsMoultonCorr3rd2`` (modules/mod_operators.py:146) read only its first five
  arguments (nonlinear/step2d.py:120-123).
"""
import ctypes
import os
import numpy as _np
from numpy import *  # noqa: F401,F403

_HERE = os.path.dirname(os.path.abspath(__file__))
_REPO = os.path.abspath(os.path.join(_HERE, "..", "..", "..", ".."))
_REF_DIR = os.path.join(_REPO, "oracle", "_ref")

GUARD = 1 << 16  # elements of zero guard on each side of every allocation


def _guarded(shape, dtype, fill):
    shape = tuple(shape) if isinstance(shape, (tuple, list)) else (int(shape),)
    n = int(_np.prod(shape)) if shape else 1
    parent = _np.zeros(n + 2 * GUARD, dtype=dtype)
    view = parent[GUARD:GUARD + n].reshape(shape)
    if fill is not None:
        view[...] = fill
    return view


def zeros(shape, dtype=_np.float64, order="C"):
    return _guarded(shape, dtype, None)


def ones(shape, dtype=_np.float64, order="C"):
    return _guarded(shape, dtype, 1)


def empty(shape, dtype=_np.float64, order="C"):
    return _guarded(shape, dtype, None)


def array(obj, dtype=None, copy=True, order="K", ndmin=0):
    a = _np.asarray(obj, dtype=dtype)
    out = _guarded(a.shape, a.dtype, None)
    out[...] = a
    return out


ndarray = _np.ndarray

# name -> parameter kinds (p pointer, d double, i int, u unsigned, b bool), in the order of
# the reference kernel signature.
_SIGS = {
    "2d": {
        "initialize": "uuupppp",
        "computeMomentumRHSPred": "pppppdd",
        "computeMomentumRHSCorr": "ppppppd",
        "computeZetaRHS": "pppppppbppip",
        "computeZetaPred": "dpppp",
        "computeMomentumPred": "dppppppppp",
        "AdamsMoultonCorr3rd": "dpppp",
        "AdamsMoultonCorr3rd2": "dppppppppppp",
    },
    "rhs": {
        "initialize": "uuupppp",
        "addCoriolis": "pppppp",
        "horizontalAdvection": "ppppppp",
        "verticalAdvection": "pppppp",
        "vertIntegral": "pp",
    },
    "step3d": {
        "initialize": "uuupppp",
        "setVerticalVelEq": "ppp",
        "omega": "ppppppp",
        "set_depth": "ippppdppppp",
        "set_zeta": "ppp",
        "setLateralUVBCs": "dpppppp",
        "set_maxflux": "ppppp",
        "step3d_UV": "pppppppppppppppp" + "iiddd",
    },
    "bc": {
        "setBC": "ppud",
        "copyBC": "pppu",
    },
}
_CT = {"p": ctypes.c_void_p, "d": ctypes.c_double, "i": ctypes.c_int, "u": ctypes.c_uint,
       "b": ctypes.c_bool}
_LIBS = {}
launch_log = []   # (module, kernel, nthreads) of every launch, for the golden generator


def _lib(mod):
    if mod not in _LIBS:
        _LIBS[mod] = ctypes.CDLL(os.path.join(_REF_DIR, "libsfref_%s.so" % mod))
    return _LIBS[mod]


def _to_c(kind, x):
    if kind == "p":
        if isinstance(x, _np.ndarray):
            return ctypes.c_void_p(x.ctypes.data)
        raise TypeError("pointer argument must be an array, got %r" % type(x))
    if kind == "d":
        return ctypes.c_double(float(x))
    if kind == "i":
        return ctypes.c_int(int(x))
    if kind == "u":
        return ctypes.c_uint(int(x) & 0xFFFFFFFF)
    if kind == "b":
        return ctypes.c_bool(bool(x))
    raise ValueError(kind)


class RawKernel:
    def __init__(self, mod, name):
        self.mod, self.name = mod, name
        self.sig = _SIGS[mod].get(name)
        if self.sig is None:        # debug kernels the step never launches (e.g. step3d_UV_test)
            return
        f = getattr(_lib(mod), "sfref_" + name)
        f.argtypes = [ctypes.c_long, ctypes.c_int] + [_CT[k] for k in self.sig]
        f.restype = None
        self.f = f

    def __call__(self, grid, block, args, **kw):
        if self.sig is None:
            raise NotImplementedError("kernel %s is not bound in the shim" % self.name)
        n = int(_np.prod(grid)) * int(_np.prod(block))
        args = tuple(args)[:len(self.sig)]
        if len(args) < len(self.sig):
            raise TypeError("%s expects %d arguments" % (self.name, len(self.sig)))
        launch_log.append((self.mod, self.name, n))
        self.f(n, 1, *[_to_c(k, a) for k, a in zip(self.sig, args)])


class RawModule:
    def __init__(self, code=None, options=(), **kw):
        if "computeZetaRHS" in code:
            self.mod = "2d"
        elif "horizontalAdvection" in code:
            self.mod = "rhs"
        elif "step3d_UV" in code:
            self.mod = "step3d"
        elif "copyBC" in code:
            self.mod = "bc"
        else:
            raise ValueError("unknown reference module")

    def get_function(self, name):
        return RawKernel(self.mod, name)


class ElementwiseKernel:
    def __init__(self, *a, **kw):
        pass

    def __call__(self, *a, **kw):
        raise NotImplementedError("ElementwiseKernel is not used on the reference's step path")


class _Cuda:
    def set_allocator(self, *a, **kw):
        pass


cuda = _Cuda()
