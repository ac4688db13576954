"""Test helpers: the two CPU checkers and comparison routines.

Checkers (test infrastructure, never the product):
  * oracle/libtlfr_oracle.so — the C restatement (oracle/tlfr_oracle.c), built by
    `make -C oracle` when missing.
  * oracle/_ref/libtlfr_ref.so (+ _m64) — the reference's own CPU code built by
    oracle/build_ref.sh; present when the reference tree was available to build it.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "libtlfr_oracle.so")
REF_LIB = os.path.join(ORACLE_DIR, "_ref", "libtlfr_ref.so")
REF_LIB_M64 = os.path.join(ORACLE_DIR, "_ref", "libtlfr_ref_m64.so")
GOLDEN = os.path.join(ROOT, "tests", "golden")

_VP = ctypes.c_void_p
_FP = ctypes.POINTER(ctypes.c_float)
_IP = ctypes.POINTER(ctypes.c_int)
_DP = ctypes.POINTER(ctypes.c_double)


def f32p(a):
    return a.ctypes.data_as(_FP)


def i32p(a):
    return a.ctypes.data_as(_IP)


_oracle = None
_refs = {}


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_LIB):
            subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
        _oracle = ctypes.CDLL(ORACLE_LIB)
        _oracle.orc_last_error.restype = ctypes.c_char_p
    return _oracle


def ref_available(m64=False):
    return os.path.exists(REF_LIB_M64 if m64 else REF_LIB)


def ref_lib(m64=False):
    path = REF_LIB_M64 if m64 else REF_LIB
    if path not in _refs:
        _refs[path] = ctypes.CDLL(path)
    return _refs[path]


class CpuRecon:
    """Common handle over the oracle restatement ('orc') or the reference build ('ref')."""

    def __init__(self, kind, records, coc, aperture=1.0, focus=1.0, uvt=None, lens=0, time=0,
                 output_spp=0, nthreads=8, m64=False, density=None):
        self.kind = kind
        rec = np.ascontiguousarray(records, np.float32)
        H, W, S = rec.shape[:3]
        self.W, self.H, self.S = W, H, S
        h = _VP()
        bs = ctypes.c_double()
        uv = (ctypes.c_float * 3)(*uvt) if uvt is not None else None
        if kind == "orc":
            self.lib = oracle_lib()
            r = self.lib.orc_create(f32p(rec), W, H, S, ctypes.c_float(coc[0]), ctypes.c_float(coc[1]),
                                    ctypes.c_float(aperture), ctypes.c_float(focus), uv, lens, time, output_spp,
                                    nthreads, ctypes.byref(h), ctypes.byref(bs))
            if r:
                raise RuntimeError(self.lib.orc_last_error())
        else:
            self.lib = ref_lib(m64)
            os.environ.setdefault("TLFR_REF_THREADS", str(nthreads))
            if density is None:
                r = self.lib.ref_create(f32p(rec), W, H, S, ctypes.c_float(coc[0]), ctypes.c_float(coc[1]),
                                        ctypes.c_float(aperture), ctypes.c_float(focus), uv, lens, time,
                                        ctypes.byref(h), ctypes.byref(bs))
            else:
                self._density = np.ascontiguousarray(density, np.float32)
                r = self.lib.ref_create_density(f32p(rec), W, H, S, ctypes.c_float(coc[0]),
                                                ctypes.c_float(coc[1]), f32p(self._density), ctypes.c_float(aperture),
                                                ctypes.c_float(focus), uv, lens, time, ctypes.byref(h),
                                                ctypes.byref(bs))
            if r:
                self.lib.ref_last_error.restype = ctypes.c_char_p
                raise RuntimeError(self.lib.ref_last_error())
        self.h = h
        self.build_seconds = bs.value
        self._info()

    def _info(self):
        n, s, root, spp, osp, hgt = (ctypes.c_int() for _ in range(6))
        cc = np.zeros(2, np.float32)
        if self.kind == "orc":
            self.lib.orc_tree_info(self.h, ctypes.byref(n), ctypes.byref(s), ctypes.byref(root), ctypes.byref(spp),
                                   f32p(cc), ctypes.byref(osp), ctypes.byref(hgt))
        else:
            self.lib.ref_tree_info(self.h, ctypes.byref(n), ctypes.byref(s), ctypes.byref(root), ctypes.byref(spp),
                                   f32p(cc), ctypes.byref(osp))
        self.num_nodes, self.num_samples, self.root = n.value, s.value, root.value
        self.spp_pow2, self.out_spp, self.coc_adjusted = spp.value, osp.value, cc.copy()

    def tree(self):
        nf = np.zeros((self.num_nodes, 14), np.float32)
        ni = np.zeros((self.num_nodes, 5), np.int32)
        sf = np.zeros((self.num_samples, 12), np.float32)
        if self.kind == "orc":
            ids = np.zeros(self.num_samples, np.int32)
            self.lib.orc_tree_export(self.h, f32p(nf), i32p(ni), f32p(sf), i32p(ids))
        else:
            ids = None
            self.lib.ref_tree_export(self.h, f32p(nf), i32p(ni), f32p(sf))
        return nf, ni, sf, ids, self.root

    def output_samples(self):
        out = np.zeros((64 * self.out_spp, 5), np.float32)
        fn = self.lib.orc_output_samples if self.kind == "orc" else self.lib.ref_output_samples
        fn(self.h, f32p(out))
        return out

    def reconstruct(self):
        img = np.zeros((self.H, self.W, 4), np.float32)
        sec = ctypes.c_double()
        st = np.zeros(16, np.float64)
        if self.kind == "orc":
            self.lib.orc_reconstruct(self.h, f32p(img), ctypes.byref(sec), st.ctypes.data_as(_DP))
        else:
            self.lib.ref_reconstruct(self.h, f32p(img), ctypes.byref(sec), None)
        self.last_seconds = sec.value
        self.last_stats = st
        return img

    def reconstruct_rows(self, y0, y1):
        img = np.zeros((y1 - y0, self.W, 4), np.float32)
        sec = ctypes.c_double()
        fn = self.lib.orc_reconstruct_rows if self.kind == "orc" else self.lib.ref_reconstruct_rows
        r = fn(self.h, y0, y1, f32p(img), ctypes.byref(sec))
        assert r == 0
        self.last_seconds = sec.value
        return img

    def reconstruct_rowlist(self, rows):
        """The listed rows, in one call (the reference build runs them in parallel)."""
        rows = [int(y) for y in rows]
        img = np.zeros((len(rows), self.W, 4), np.float32)
        if self.kind == "ref":
            r = np.asarray(rows, np.int32)
            sec = ctypes.c_double()
            assert self.lib.ref_reconstruct_rowlist(self.h, i32p(r), len(rows), f32p(img), ctypes.byref(sec)) == 0
            self.last_seconds = sec.value
        else:
            t = 0.0
            for k, y in enumerate(rows):
                img[k] = self.reconstruct_rows(y, y + 1)[0]
                t += self.last_seconds
            self.last_seconds = t
        return img

    def set_view(self, params):
        """The camera fields of a tlfr.CameraParams into the reference's CameraParams."""
        assert self.kind == "ref"
        m = [np.ascontiguousarray(x, np.float32).reshape(16) for x in
             (params.projection, params.cameraToWorld, params.worldToCamera)]
        assert self.lib.ref_set_view(self.h, f32p(m[0]), f32p(m[1]), f32p(m[2]), ctypes.c_float(params.far),
                                     int(params.windowSize[0]), int(params.windowSize[1]),
                                     ctypes.c_float(params.apertureRadius), ctypes.c_float(params.focusDistance)) == 0
        self._views = m

    def dof_motion_shadows(self, light):
        """TreeGather::reconstructDofMotionShadows of the reference build: this handle is the
        camera's, light the light's (views set with set_view); returns the image [H, W, 4]."""
        assert self.kind == "ref"
        out = np.zeros((self.H, self.W, 4), np.float32)
        assert self.lib.ref_reconstruct_dof_motion_shadows(self.h, light.h, f32p(out)) == 0
        return out

    def shadows(self, queries, density):
        """TreeGather::reconstructShadows of the reference build: queries [H, W, qspp, 16],
        density [H, W, qspp]; returns the query buffer's colours [H, W, qspp, 4]."""
        assert self.kind == "ref"
        q = np.ascontiguousarray(queries, np.float32)
        d = np.ascontiguousarray(density, np.float32)
        out = np.zeros(q.shape[:3] + (4,), np.float32)
        assert self.lib.ref_reconstruct_shadows(self.h, f32p(q), q.shape[2], f32p(d), f32p(out)) == 0
        return out

    def gpu_toggle_image(self):
        """The reference's CPU restatement of its GPU-toggle algorithm over the whole
        image (CudaReconstruction::reconstructCPU, reference build only)."""
        assert self.kind == "ref"
        img = np.zeros((self.H, self.W, 4), np.float32)
        sec = ctypes.c_double()
        assert self.lib.ref_gpu_toggle_image(self.h, f32p(img), ctypes.byref(sec)) == 0
        self.last_seconds = sec.value
        return img

    def gpu_toggle_queries(self, xyi):
        """Output samples (x, y, i) through CudaReconstruction::reconstructCPUSingle."""
        assert self.kind == "ref"
        q = np.ascontiguousarray(np.asarray(xyi, np.int32).reshape(-1, 3))
        out = np.zeros((len(q), 4), np.float32)
        assert self.lib.ref_gpu_toggle_queries(self.h, i32p(q), len(q), f32p(out)) == 0
        return out

    def query(self, x, y, i, cap=1 << 16):
        rgba = np.zeros(4, np.float32)
        tr = np.zeros(cap, np.int32)
        fn = self.lib.orc_query if self.kind == "orc" else self.lib.ref_query
        n = fn(self.h, x, y, i, f32p(rgba), i32p(tr), cap)
        return rgba, tr[:n].copy()

    def close(self):
        if self.h:
            (self.lib.orc_destroy if self.kind == "orc" else self.lib.ref_destroy)(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def canonical_tree(tree):
    """DFS (child0 first) serialisation of a hierarchy: per node its bounds bits,
    sample count and, for leaves, the sample records' bits in order.  Node
    numbering does not enter, so trees built in a different emission order compare
    equal when their structure, bounds and samples do."""
    nf, ni, sf, _ids, root = tree
    out = []
    stack = [root]
    while stack:
        i = stack.pop()
        leaf = ni[i, 0] == -1
        rec = [nf[i].view(np.uint32).tobytes(), int(leaf)]
        if leaf:
            s0, s1 = int(ni[i, 2]), int(ni[i, 3])
            rec.append(sf[s0:s1, :11].view(np.uint32).tobytes())
        else:
            stack.append(int(ni[i, 1]))
            stack.append(int(ni[i, 0]))
        out.append(rec)
    return out


def tree_digest(tree):
    h = hashlib.sha256()
    n = 0
    for rec in canonical_tree(tree):
        for part in rec:
            h.update(part if isinstance(part, bytes) else str(part).encode())
        n += 1
    return h.hexdigest(), n


def compare_trees(a, b, max_report=3):
    """Returns a list of mismatch descriptions (empty when identical)."""
    ca, cb = canonical_tree(a), canonical_tree(b)
    msgs = []
    if len(ca) != len(cb):
        msgs.append(f"reachable node count {len(ca)} vs {len(cb)}")
    for k, (x, y) in enumerate(zip(ca, cb)):
        if x != y:
            msgs.append(f"node {k} (dfs order) differs")
            if len(msgs) >= max_report:
                break
    return msgs


def sample_queries(W, H, M, n, seed=0):
    rng = np.random.default_rng(seed)
    return np.stack([rng.integers(0, W, n), rng.integers(0, H, n), rng.integers(0, M, n)], 1).astype(np.int32)


def rel_err(a, b, floor=1e-6):
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


def hash_pattern(x, y):
    """Output pattern of pixel (x, y): hashBits(x, y) % 64 (Hash.hpp:169-183,
    Reconstruction.cpp:653)."""
    m = 0xffffffff
    a, b, c = x & m, y & m, 0x9e3779b9
    a = (a - b) & m; a = (a - c) & m; a ^= (c >> 13)
    b = (b - c) & m; b = (b - a) & m; b = (b ^ (a << 8)) & m
    c = (c - a) & m; c = (c - b) & m; c ^= (b >> 13)
    a = (a - b) & m; a = (a - c) & m; a ^= (c >> 12)
    b = (b - c) & m; b = (b - a) & m; b = (b ^ (a << 16)) & m
    c = (c - a) & m; c = (c - b) & m; c ^= (b >> 5)
    a = (a - b) & m; a = (a - c) & m; a ^= (c >> 3)
    b = (b - c) & m; b = (b - a) & m; b = (b ^ (a << 10)) & m
    c = (c - a) & m; c = (c - b) & m; c ^= (b >> 15)
    return c % 64
