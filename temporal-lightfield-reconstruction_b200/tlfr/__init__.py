"""Python binding of libtlfr.so, the B200 temporal light field reconstruction library.

Mirrors the reference reconstruction library's interface
(reference src/reconstruction_lib):

    UVTSampleBuffer(path)                     common/SampleBuffer.cpp:230-387
    UVTSampleBuffer.serialize(...)            common/SampleBuffer.cpp:404-564
    CameraParams                              common/CameraParams.hpp:74-107
    TreeGather(sbuf, params, aperture, focus) reconstruction/Reconstruction.hpp:45
    TreeGather.reconstructDofMotion(image)    reconstruction/Reconstruction.cpp:221-295

The library computes on the GPU only.  Loading fails loudly when libtlfr.so is
missing; calls fail with TlfrError (status + message) when there is no CUDA
device.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libtlfr.so")

STATUS = {
    0: "TLFR_OK", 1: "TLFR_BAD_ARG", 2: "TLFR_IO", 3: "TLFR_FORMAT", 4: "TLFR_OOM",
    5: "TLFR_CUDA", 6: "TLFR_OVERFLOW", 7: "TLFR_TIMEOUT", 8: "TLFR_NO_DEVICE", 9: "TLFR_EMPTY",
}

SCENE_PLANES, SCENE_CARDS, SCENE_CARDS_LARGE = 0, 1, 2
LENS_BOX, LENS_GAUSSIAN = 0, 1
TIME_BOX, TIME_GAUSSIAN = 0, 1


class TlfrError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class _Params(ctypes.Structure):
    _fields_ = [
        ("aperture_adjust", ctypes.c_float),
        ("focus_adjust", ctypes.c_float),
        ("lens_filter", ctypes.c_int),
        ("time_filter", ctypes.c_int),
        ("override_uvt", ctypes.c_int),
        ("uvt", ctypes.c_float * 3),
        ("output_spp", ctypes.c_int),
        ("device", ctypes.c_int),
        ("enable_cuda", ctypes.c_int),
    ]


class Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "num_output_samples", "num_leaf_nodes", "num_samples_in_leaf_nodes", "num_samples_within_1r",
        "num_samples_fetched", "num_surfaces", "num_2r", "num_surfaces_merged", "num_at_least_one",
        "num_overflow_queries", "num_empty", "build_ms", "query_ms", "query_kernel_ms", "build_launches",
        "query_launches", "overflow_leaves", "overflow_stack", "overflow_surfaces", "overflow_samples",
        "num_heavy_queries", "light_ms", "heavy_ms", "num_retried_queries")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


_lib = None
_VP = ctypes.c_void_p
_FP = ctypes.POINTER(ctypes.c_float)
_IP = ctypes.POINTER(ctypes.c_int)


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libtlfr.so (built by __graft_entry__.build() or `make` in the package)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libtlfr.so not found at {path}; build it with `make -C {os.path.dirname(path)}`")
    lib = ctypes.CDLL(path)
    sig = {
        "tlfr_params_default": (None, [ctypes.POINTER(_Params)]),
        "tlfr_buffer_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_VP)]),
        "tlfr_buffer_from_host": (ctypes.c_int, [_FP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                                 ctypes.c_float, ctypes.POINTER(_VP)]),
        "tlfr_buffer_save": (ctypes.c_int, [_VP, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]),
        "tlfr_buffer_info": (ctypes.c_int, [_VP, _IP, _IP, _IP, _FP, _FP]),
        "tlfr_buffer_records": (_FP, [_VP]),
        "tlfr_buffer_free": (None, [_VP]),
        "tlfr_create": (ctypes.c_int, [_VP, ctypes.POINTER(_Params), _VP, ctypes.POINTER(_VP)]),
        "tlfr_create_device": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                              ctypes.c_float, ctypes.POINTER(_Params), _VP, ctypes.POINTER(_VP)]),
        "tlfr_rebuild_device": (ctypes.c_int, [_VP, _VP]),
        "tlfr_rebuild": (ctypes.c_int, [_VP, _VP]),
        "tlfr_reconstruct": (ctypes.c_int, [_VP, _VP, ctypes.c_int, ctypes.POINTER(Stats)]),
        "tlfr_set_output": (ctypes.c_int, [_VP, ctypes.POINTER(_Params)]),
        "tlfr_sync": (ctypes.c_int, [_VP]),
        "tlfr_trim": (ctypes.c_int, [_VP]),
        "tlfr_get_stats": (ctypes.c_int, [_VP, ctypes.POINTER(Stats)]),
        "tlfr_destroy": (None, [_VP]),
        "tlfr_last_error": (ctypes.c_char_p, [_VP]),
        "tlfr_tree_info": (ctypes.c_int, [_VP, _IP, _IP, _IP, _IP]),
        "tlfr_tree_export": (ctypes.c_int, [_VP, _FP, _IP, _FP, _IP]),
        "tlfr_output_samples": (ctypes.c_int, [_VP, _FP]),
        "tlfr_trace_queries": (ctypes.c_int, [_VP, _IP, ctypes.c_int, _FP, _IP, ctypes.c_int]),
        "tlfr_query_samples_noalloc": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _VP, _VP]),
        "tlfr_output_sample_buffer": (ctypes.c_int, [_VP, ctypes.POINTER(_VP)]),
        "tlfr_reconstruct_shadows": (ctypes.c_int, [_VP, _FP, ctypes.c_int, _FP, _FP]),
        "tlfr_reconstruct_dof_motion_shadows": (ctypes.c_int, [_VP, ctypes.POINTER(_View), _FP, _VP,
                                                               ctypes.POINTER(_View), _FP, ctypes.c_int]),
        "tlfr_synth_scene": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_ulonglong, _FP, _FP]),
        "tlfr_synth_reference_image": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                      ctypes.c_ulonglong, _FP]),
        "tlfr_route_features": (ctypes.c_int, [_VP, _VP]),
        "tlfr_route_labels": (ctypes.c_int, [_VP, ctypes.c_float, _VP, _VP]),
        "tlfr_route_labels_ref": (ctypes.c_int, [_VP, _VP, ctypes.c_float, _VP, _VP]),
        "tlfr_router_create": (ctypes.c_int, [ctypes.c_int, _VP, ctypes.c_uint, _FP, _FP, ctypes.POINTER(_VP)]),
        "tlfr_router_destroy": (None, [_VP]),
        "tlfr_router_last_error": (ctypes.c_char_p, [_VP]),
        "tlfr_router_num_params": (ctypes.c_int, []),
        "tlfr_router_train": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                             ctypes.c_uint, _FP]),
        "tlfr_router_gradient": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_int, _FP, _FP]),
        "tlfr_router_predict": (ctypes.c_int, [_VP, _VP, ctypes.c_longlong, _VP]),
        "tlfr_router_get_params": (ctypes.c_int, [_VP, _FP]),
        "tlfr_router_set_params": (ctypes.c_int, [_VP, _FP]),
        "tlfr_set_routing": (ctypes.c_int, [_VP, _VP, ctypes.c_float]),
        "tlfr_batch_create": (ctypes.c_int, [ctypes.POINTER(_VP), ctypes.c_int, ctypes.POINTER(_VP), _VP,
                                             ctypes.c_int, ctypes.POINTER(_VP)]),
        "tlfr_batch_run": (ctypes.c_int, [_VP]),
        "tlfr_batch_sync": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_double)]),
        "tlfr_batch_info": (ctypes.c_int, [_VP, _IP]),
        "tlfr_batch_layout": (ctypes.c_int, [_VP, _IP, ctypes.POINTER(ctypes.c_longlong)]),
        "tlfr_batch_create_frames": (ctypes.c_int, [_VP, ctypes.c_int, _VP, ctypes.c_int, ctypes.c_size_t,
                                                    ctypes.POINTER(_VP)]),
        "tlfr_batch_last_error": (ctypes.c_char_p, [_VP]),
        "tlfr_batch_destroy": (None, [_VP]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _f32p(a: np.ndarray):
    return a.ctypes.data_as(_FP)


def _i32p(a: np.ndarray):
    return a.ctypes.data_as(_IP)


def _check(status: int, ctx=None):
    if status != 0:
        msg = load_library().tlfr_last_error(ctx)
        raise TlfrError(status, msg.decode() if msg else "")


def synth_scene(preset: int, width: int, height: int, spp: int, seed: int = 1):
    """Seeded analytic scene -> (records float32 [H, W, spp, 16], (C0, C1))."""
    lib = load_library()
    rec = np.empty((height, width, spp, 16), np.float32)
    coc = np.zeros(2, np.float32)
    _check(lib.tlfr_synth_scene(preset, width, height, spp, seed, _f32p(rec), _f32p(coc)))
    return rec, (float(coc[0]), float(coc[1]))


def synth_reference_image(preset: int, width: int, height: int, samples: int = 1024, seed: int = 1) -> np.ndarray:
    """Ground-truth RGBA image [H, W, 4] of the seeded scene: the mean colour
    over `samples` points per pixel spread over the pixel, the unit lens disk
    and the shutter (computed on the current CUDA device)."""
    lib = load_library()
    img = np.empty((height, width, 4), np.float32)
    _check(lib.tlfr_synth_reference_image(preset, width, height, samples, seed, _f32p(img)))
    return img


class UVTSampleBuffer:
    """Host sample buffer: W*H*spp records of 16 floats (SampleBuffer.cpp:283-286)."""

    def __init__(self, path: Optional[str] = None, *, records=None, coc=None, width=None, height=None, spp=None):
        lib = load_library()
        h = _VP()
        if path is not None:
            _check(lib.tlfr_buffer_load(os.fsencode(path), ctypes.byref(h)))
        else:
            rec = np.ascontiguousarray(records, dtype=np.float32)
            if width is None:
                height, width, spp = rec.shape[:3]
            _check(lib.tlfr_buffer_from_host(_f32p(rec), width, height, spp, coc[0], coc[1], ctypes.byref(h)))
        self._h = h

    @classmethod
    def _from_handle(cls, h) -> "UVTSampleBuffer":
        b = cls.__new__(cls)
        b._h = h
        return b

    @property
    def handle(self):
        return self._h

    def info(self):
        W, H, S = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        c0, c1 = ctypes.c_float(), ctypes.c_float()
        _check(load_library().tlfr_buffer_info(self._h, ctypes.byref(W), ctypes.byref(H), ctypes.byref(S),
                                               ctypes.byref(c0), ctypes.byref(c1)))
        return W.value, H.value, S.value, (c0.value, c1.value)

    def getWidth(self):
        return self.info()[0]

    def getHeight(self):
        return self.info()[1]

    def getCocCoeffs(self):
        return self.info()[3]

    def records(self) -> np.ndarray:
        W, H, S, _ = self.info()
        p = load_library().tlfr_buffer_records(self._h)
        return np.ctypeslib.as_array(p, shape=(H, W, S, 16)).copy()

    def serialize(self, path: str, separate_header: bool = False, binary: bool = False):
        _check(load_library().tlfr_buffer_save(self._h, os.fsencode(path), int(separate_header), int(binary)))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.tlfr_buffer_free(self._h)
            self._h = None


class _View(ctypes.Structure):
    _fields_ = [("projection", ctypes.c_float * 16), ("camera_to_world", ctypes.c_float * 16),
                ("world_to_camera", ctypes.c_float * 16), ("far_plane", ctypes.c_float),
                ("window_size", ctypes.c_int * 2), ("aperture_radius", ctypes.c_float),
                ("focus_distance", ctypes.c_float)]


def _identity():
    return np.eye(4, dtype=np.float32)


@dataclass
class CameraParams:
    """The CameraParams fields the reconstruction path reads (CameraParams.hpp:74-107).

    enableCuda is the reference's CPU/GPU toggle (CameraParams.hpp:88): False (its
    default) selects the algorithm of the reference's CPU reconstruction
    (TreeGather::Filterer), True the algorithm of its GPU reconstruction
    (ReconstructionCuda.cpp / ReconstructionCudaKernels.cu).  This library runs
    both on the GPU.  overrideUVT: None or (u, v, t); the t=1 pinhole image is
    (0, 0, 1) (reconstruction_app/App.cpp:450).
    """
    lensFilter: int = LENS_BOX
    timeFilter: int = TIME_BOX
    overrideUVT: Optional[Tuple[float, float, float]] = None
    enableCuda: bool = False
    outputSpp: int = 0          # 0: reference default (128, or 1 with overrideUVT)
    device: int = 0
    # the camera, read only by the shadowed reconstruction (CameraParams.hpp:96-104;
    # CameraControls getCameraToWorld / getWorldToCamera / getFar): 4x4 matrices
    projection: np.ndarray = field(default_factory=_identity)
    cameraToWorld: np.ndarray = field(default_factory=_identity)
    worldToCamera: np.ndarray = field(default_factory=_identity)
    far: float = 3.0
    windowSize: Tuple[int, int] = (0, 0)
    apertureRadius: float = 0.0
    focusDistance: float = 1.0

    def _view(self) -> _View:
        v = _View()
        for name, m in (("projection", self.projection), ("camera_to_world", self.cameraToWorld),
                        ("world_to_camera", self.worldToCamera)):
            a = np.ascontiguousarray(m, np.float32).reshape(16)
            getattr(v, name)[:] = [float(x) for x in a]
        v.far_plane = self.far
        v.window_size[0], v.window_size[1] = int(self.windowSize[0]), int(self.windowSize[1])
        v.aperture_radius = self.apertureRadius
        v.focus_distance = self.focusDistance
        return v

    def _to_c(self, aperture: float, focus: float) -> _Params:
        p = _Params()
        load_library().tlfr_params_default(ctypes.byref(p))
        p.aperture_adjust = aperture
        p.focus_adjust = focus
        p.lens_filter = self.lensFilter
        p.time_filter = self.timeFilter
        if self.overrideUVT is not None:
            p.override_uvt = 1
            p.uvt[0], p.uvt[1], p.uvt[2] = self.overrideUVT
        p.output_spp = self.outputSpp
        p.device = self.device
        p.enable_cuda = 1 if self.enableCuda else 0
        return p


class TreeGather:
    """Hierarchy build + reconstruction (reconstruction/Reconstruction.hpp:42-48)."""

    def __init__(self, sbuf: Optional[UVTSampleBuffer], params: Optional[CameraParams] = None,
                 apertureAdjust: float = 1.0, focalDistanceAdjust: float = 1.0, *, stream: int = 0,
                 device_records=None):
        lib = load_library()
        self.params = params or CameraParams()
        p = self.params._to_c(apertureAdjust, focalDistanceAdjust)
        h = _VP()
        if device_records is not None:
            ptr, (W, H, S), (c0, c1) = device_records
            _check(lib.tlfr_create_device(_VP(ptr), W, H, S, c0, c1, ctypes.byref(p), _VP(stream), ctypes.byref(h)))
            self.size = (W, H)
        else:
            _check(lib.tlfr_create(sbuf.handle, ctypes.byref(p), _VP(stream), ctypes.byref(h)))
            self.size = sbuf.info()[:2]
        self._h = h

    @property
    def handle(self):
        return self._h

    def reconstructDofMotion(self, image: Optional[np.ndarray] = None, stats: bool = False):
        """RGBA float32 image [H, W, 4]; with stats=True returns (image, Stats)."""
        W, H = self.size
        if image is None:
            image = np.empty((H, W, 4), np.float32)
        st = Stats()
        _check(load_library().tlfr_reconstruct(self._h, image.ctypes.data, 0, ctypes.byref(st) if stats else None),
               self._h)
        return (image, st) if stats else image

    def reconstruct_to_device(self, dev_ptr: int, stats: bool = False):
        st = Stats()
        _check(load_library().tlfr_reconstruct(self._h, _VP(dev_ptr), 1, ctypes.byref(st) if stats else None),
               self._h)
        return st if stats else None

    def rebuild(self, dev_ptr: int):
        """Rebuild the hierarchy from device records of the same size."""
        _check(load_library().tlfr_rebuild_device(self._h, _VP(dev_ptr)), self._h)

    def rebuild_from(self, sbuf: "UVTSampleBuffer"):
        """Upload a host buffer of the same size and rebuild the hierarchy."""
        _check(load_library().tlfr_rebuild(self._h, sbuf.handle), self._h)

    def trim(self):
        """Free the hierarchy build's working storage (the hierarchy stays)."""
        _check(load_library().tlfr_trim(self._h), self._h)

    def set_output(self, params: CameraParams):
        p = params._to_c(1.0, 1.0)
        _check(load_library().tlfr_set_output(self._h, ctypes.byref(p)), self._h)
        self.params = params

    def stats(self) -> Stats:
        st = Stats()
        _check(load_library().tlfr_get_stats(self._h, ctypes.byref(st)), self._h)
        return st

    def tree_info(self):
        n, s, r, h = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(load_library().tlfr_tree_info(self._h, ctypes.byref(n), ctypes.byref(s), ctypes.byref(r),
                                             ctypes.byref(h)), self._h)
        return n.value, s.value, r.value, h.value

    def tree_export(self):
        n, s, r, _ = self.tree_info()
        nodef = np.zeros((n, 14), np.float32)
        nodei = np.zeros((n, 5), np.int32)
        samplef = np.zeros((s, 12), np.float32)
        ids = np.zeros(s, np.int32)
        _check(load_library().tlfr_tree_export(self._h, _f32p(nodef), _i32p(nodei), _f32p(samplef), _i32p(ids)),
               self._h)
        return nodef, nodei, samplef, ids, r

    def output_samples(self) -> np.ndarray:
        n = load_library().tlfr_output_samples(self._h, None)
        out = np.zeros((n, 5), np.float32)
        load_library().tlfr_output_samples(self._h, _f32p(out))
        return out

    def reconstructShadows(self, queries: np.ndarray, density: Optional[np.ndarray] = None) -> np.ndarray:
        """TreeGather::reconstructShadows (Reconstruction.cpp:302-344) for light-space query
        records [..., 16]: per query the shadowed colour RGBA (the reference writes it into
        the query buffer's sample colours)."""
        q = np.ascontiguousarray(queries, np.float32).reshape(-1, 16)
        n = q.shape[0]
        out = np.zeros((n, 4), np.float32)
        dp = None
        if density is not None:
            d = np.ascontiguousarray(density, np.float32).reshape(-1)
            assert d.size == n
            dp = _f32p(d)
        _check(load_library().tlfr_reconstruct_shadows(self._h, _f32p(q), n, dp, _f32p(out)), self._h)
        return out.reshape(tuple(np.shape(queries)[:-1]) + (4,))

    def reconstructDofMotionShadows(self, shadowTG: "TreeGather",
                                    density: Optional[np.ndarray] = None) -> np.ndarray:
        """TreeGather::reconstructDofMotionShadows (Reconstruction.cpp:355-433): this
        hierarchy is the camera's, shadowTG's the light's (same image size); the views come
        from the two TreeGathers' CameraParams.  density: the camera buffer's
        LIGHTSPACE_DENSITY channel, one float per input record ([H, W, spp] or flat), or None
        for 1.  Returns the image [H, W, 4]."""
        W, H = self.size
        out = np.zeros((H, W, 4), np.float32)
        dp = None
        if density is not None:
            d = np.ascontiguousarray(density, np.float32).reshape(-1)
            dp = _f32p(d)
        cv, lv = self.params._view(), shadowTG.params._view()
        _check(load_library().tlfr_reconstruct_dof_motion_shadows(self._h, ctypes.byref(cv), dp, shadowTG._h,
                                                                   ctypes.byref(lv), _f32p(out), 0), self._h)
        return out

    def output_sample_buffer(self) -> "UVTSampleBuffer":
        """The last reconstruction's output samples as a sample buffer (the reference's
        m_obuf dump, Reconstruction.cpp:290-294, 696-712)."""
        h = _VP()
        _check(load_library().tlfr_output_sample_buffer(self._h, ctypes.byref(h)), self._h)
        return UVTSampleBuffer._from_handle(h)

    def trace_queries(self, xyi: Sequence[Tuple[int, int, int]], stride: int = 4096):
        q = np.ascontiguousarray(np.asarray(xyi, np.int32).reshape(-1, 3))
        n = q.shape[0]
        rgba = np.zeros((n, 4), np.float32)
        trace = np.zeros((n, stride), np.int32)
        _check(load_library().tlfr_trace_queries(self._h, _i32p(q), n, _f32p(rgba), _i32p(trace), stride), self._h)
        return rgba, trace

    def route_features(self, d_feats: int):
        """Eight routing features per pixel into device memory (W*H*8 floats)."""
        _check(load_library().tlfr_route_features(self._h, _VP(d_feats)), self._h)

    def route_labels(self, d_labels: int, d_rgba: int, tol: float = 0.01, d_ref: Optional[int] = None):
        """Plain reconstruction into d_rgba plus every pixel's label: the fast path within tol of
        the plain pixel, or (d_ref, a device ground-truth image) a squared error against d_ref
        at most tol above the plain pixel's."""
        if d_ref is None:
            _check(load_library().tlfr_route_labels(self._h, tol, _VP(d_labels), _VP(d_rgba)), self._h)
        else:
            _check(load_library().tlfr_route_labels_ref(self._h, _VP(d_ref), tol, _VP(d_labels), _VP(d_rgba)),
                   self._h)

    def set_routing(self, router: Optional["Router"], threshold: float = 0.8):
        """Learned routing on (router) or off (None) for the following reconstructions."""
        _check(load_library().tlfr_set_routing(self._h, router.handle if router else None, threshold), self._h)
        self._router = router

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.tlfr_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class Router:
    """The learned single-surface router (8-64-64-1 MLP on the tensor cores)."""

    NUM_FEATURES = 8

    def __init__(self, device: int = 0, seed: int = 1, mean=None, inv_std=None, stream: int = 0):
        lib = load_library()
        h = _VP()
        m = np.ascontiguousarray(mean, np.float32) if mean is not None else None
        s = np.ascontiguousarray(inv_std, np.float32) if inv_std is not None else None
        st = lib.tlfr_router_create(device, _VP(stream), seed, _f32p(m) if m is not None else None,
                                    _f32p(s) if s is not None else None, ctypes.byref(h))
        if st != 0:
            raise TlfrError(st, (lib.tlfr_router_last_error(None) or b"").decode())
        self._h = h

    @property
    def handle(self):
        return self._h

    def _ok(self, st):
        if st != 0:
            raise TlfrError(st, (load_library().tlfr_router_last_error(self._h) or b"").decode())

    def train(self, d_feats: int, d_labels: int, n: int, steps: int, batch: int = 8192, lr: float = 2e-3,
              seed: int = 7) -> float:
        loss = ctypes.c_float()
        self._ok(load_library().tlfr_router_train(self._h, _VP(d_feats), _VP(d_labels), n, steps, batch, lr, seed,
                                                  ctypes.byref(loss)))
        return loss.value

    def gradient(self, d_feats: int, d_labels: int, n: int):
        g = np.zeros(self.num_params(), np.float32)
        loss = ctypes.c_float()
        self._ok(load_library().tlfr_router_gradient(self._h, _VP(d_feats), _VP(d_labels), n, _f32p(g),
                                                     ctypes.byref(loss)))
        return g[:self.num_trainable()], loss.value

    def predict(self, d_feats: int, n: int, d_prob: int):
        self._ok(load_library().tlfr_router_predict(self._h, _VP(d_feats), n, _VP(d_prob)))

    @staticmethod
    def num_params() -> int:
        return load_library().tlfr_router_num_params()

    @staticmethod
    def num_trainable() -> int:
        return Router.num_params() - 2 * Router.NUM_FEATURES

    def params(self) -> np.ndarray:
        p = np.zeros(self.num_params(), np.float32)
        self._ok(load_library().tlfr_router_get_params(self._h, _f32p(p)))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.num_params()
        self._ok(load_library().tlfr_router_set_params(self._h, _f32p(p)))

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.tlfr_router_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class _BatchFrame(ctypes.Structure):
    _fields_ = [("ctx", _VP), ("output", ctypes.POINTER(_Params)), ("d_rgba", _VP)]


TILE_SHAPES = ["4x2 px x 4 samples", "8x4 px x 1 sample", "4x4 px x 2 samples", "2x2 px x 8 samples",
               "2x1 px x 16 samples"]


class Batch:
    """Frames reconstructed together as one CUDA graph (tlfr_batch_*): built
    TreeGather contexts, each with its own output settings or with an output
    setting of the frame's own (a sweep over one hierarchy: pass the same tree
    with different CameraParams)."""

    def __init__(self, trees: Sequence["TreeGather"], outputs: Sequence[int], stream: int = 0, autotune: bool = True,
                 params: Optional[Sequence[Optional["CameraParams"]]] = None, budget_bytes: int = 0):
        lib = load_library()
        n = len(trees)
        self._trees = list(trees)
        self._params = [p._to_c(1.0, 1.0) if p is not None else None for p in (params or [None] * n)]
        frames = (_BatchFrame * n)()
        for i in range(n):
            frames[i].ctx = trees[i].handle
            frames[i].output = ctypes.pointer(self._params[i]) if self._params[i] is not None else None
            frames[i].d_rgba = _VP(outputs[i])
        h = _VP()
        st = lib.tlfr_batch_create_frames(frames, n, _VP(stream), 1 if autotune else 0, ctypes.c_size_t(budget_bytes),
                                          ctypes.byref(h))
        if st != 0:
            raise TlfrError(st, (lib.tlfr_batch_last_error(None) or b"").decode())
        self._h = h
        self.n = n

    def _ok(self, st):
        if st != 0:
            raise TlfrError(st, (load_library().tlfr_batch_last_error(self._h) or b"").decode())

    def run(self):
        self._ok(load_library().tlfr_batch_run(self._h))

    def sync(self) -> float:
        ms = ctypes.c_double()
        self._ok(load_library().tlfr_batch_sync(self._h, ctypes.byref(ms)))
        return ms.value

    def tile_shapes(self):
        """The light-pass tile shape chosen per frame (index into TILE_SHAPES)."""
        b = np.zeros(self.n, np.int32)
        self._ok(load_library().tlfr_batch_info(self._h, _i32p(b)))
        return b

    def layout(self):
        """(chunk of each frame, kernel launches of one run)."""
        c = np.zeros(self.n, np.int32)
        nl = ctypes.c_longlong()
        self._ok(load_library().tlfr_batch_layout(self._h, _i32p(c), ctypes.byref(nl)))
        return c, nl.value

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.tlfr_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def parse_trace(row: np.ndarray):
    """Trace ints -> (flags, [(minIndex, [sample indices]), ...]); None if truncated."""
    flags, ns = int(row[0]), int(row[1])
    if ns < 0:
        return None
    k, surfaces = 2, []
    for _ in range(ns):
        n, mi = int(row[k]), int(row[k + 1])
        surfaces.append((mi, [int(v) for v in row[k + 2:k + 2 + n]]))
        k += 2 + n
    return flags, surfaces
