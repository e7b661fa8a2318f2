"""Import shims that let the reference package ``mr_recon`` run on CPU tensors.

Used only by ``make_golden.py`` in a container that has the reference source
tree. The reference package's ``__init__`` and module headers import several
GPU or plotting libraries that the KB-NUFFT path never calls (cupy, sigpy,
cufinufft, torchkbnufft, fast_pytorch_kmeans, pyeyes, turtle, cycler). Each is
replaced by a stub module; ``sigpy.fourier._get_oversamp_shape`` keeps its
real meaning because ``triton_nufft.adjoint_grid_only``
(src/mr_recon/fourier.py:538) calls it.
"""

import math
import os
import sys
import types


def _stub(name, **attrs):
    mod = types.ModuleType(name)
    for k, v in attrs.items():
        setattr(mod, k, v)
    sys.modules[name] = mod
    return mod


class _Never:
    """A class no real object is an instance of."""


class _Anything:
    def __init__(self, *a, **k):
        pass

    def __call__(self, *a, **k):
        raise RuntimeError("stubbed reference dependency called")


def install(ref_src):
    os.environ.setdefault("TORCH_COMPILE_DISABLE", "1")

    def _get_oversamp_shape(shape, ndim, oversamp):
        return list(shape)[:-ndim] + [math.ceil(oversamp * i) for i in shape[-ndim:]]

    cupy = _stub("cupy", ndarray=_Never, cuda=types.SimpleNamespace(Device=_Anything))
    cupy.get_array_module = lambda *a, **k: None
    _stub("cupyx")
    _stub("cupyx.scipy")
    _stub("cupyx.scipy.ndimage", map_coordinates=_Anything())
    sp = _stub("sigpy", get_device=_Anything(), resize=_Anything(),
               to_device=_Anything(), Device=_Anything, cpu_device=None)
    sp.fourier = _stub("sigpy.fourier", _get_oversamp_shape=_get_oversamp_shape,
                       _scale_coord=_Anything())
    sp.mri = _stub("sigpy.mri", pipe_menon_dcf=_Anything())
    sp.interp = _stub("sigpy.interp")
    sp.util = _stub("sigpy.util")
    sp.linop = _stub("sigpy.linop")
    sp.app = _stub("sigpy.app")
    _stub("cufinufft")
    _stub("torchkbnufft", KbNufft=_Anything, KbNufftAdjoint=_Anything)
    _stub("fast_pytorch_kmeans", KMeans=_Anything)
    _stub("pyeyes", ComparativeViewer=_Anything)
    _stub("turtle", forward=_Anything())
    _stub("cycler", V=None)
    if ref_src not in sys.path:
        sys.path.insert(0, ref_src)
