"""Python binding of libnsx (ctypes over the C ABI of include/nsx.h).

This mirrors the reference's hot-path interface: a ``Solver`` is what the
reference's Lnz_TRD sets up (src/NuLnz/NuCoreX.f90:807-1367), ``matvec`` is its
multiplyx/multiplya/multiplyb sequence (NuCoreX.f90:76-226) and ``solve`` its
Lnz_OP (NuCoreX.f90:240-751).  The CUDA library is the only implementation:
if libnsx.so is missing or fails to load, every entry point raises -- there is
no CPU fallback.
"""
import ctypes as C
import json
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnsx.so")

NSX_FP64 = 0
NSX_FP32 = 1
NSX_FP32_AUTO, NSX_FP32_FUSED, NSX_FP32_TC, NSX_FP32_SIMT = 0, 1, 2, 3
_ERRNAMES = {-1: "NSX_E_ARG", -2: "NSX_E_IO", -3: "NSX_E_CUDA", -4: "NSX_E_NOMEM", -5: "NSX_E_NUMERIC",
             -6: "NSX_E_NOCONV"}

_p = C.POINTER


class Species(C.Structure):
    _fields_ = [("nspart", C.c_int32), ("minJ2", C.c_int32), ("maxJ2", C.c_int32), ("njt", _p(C.c_int32)),
                ("parity", _p(C.c_int32)), ("shell_first", C.c_int32), ("nshell", C.c_int32),
                ("nkeys", C.c_int32), ("keys", _p(C.c_uint8)), ("val_off", _p(C.c_int64)),
                ("vals", _p(C.c_double)), ("words", C.c_int32), ("masks", _p(C.c_uint32)),
                ("nseg", C.c_int32), ("seg_J2", _p(C.c_int32)), ("seg_np", _p(C.c_int32)),
                ("seg_npr", _p(C.c_int32)), ("seg_off", _p(C.c_int64)), ("seg_vals", _p(C.c_double)),
                ("occ", _p(C.c_int16))]


class Problem(C.Structure):
    _fields_ = [("J2", C.c_int32), ("parity", C.c_int32), ("a", Species), ("b", Species), ("nop", C.c_int32),
                ("op_keys", _p(C.c_uint8)), ("op_vals", _p(C.c_double)), ("renorm", C.c_double)]


class Params(C.Structure):
    _fields_ = [("nev", C.c_int32), ("max_iter", C.c_int32), ("window", C.c_int32), ("keep", C.c_int32),
                ("tol", C.c_double), ("precision", C.c_int32), ("pre_iter", C.c_int32), ("seed", C.c_uint64),
                ("start", _p(C.c_double)), ("refine", C.c_int32)]


class Report(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("matvecs", C.c_int32), ("restarts", C.c_int32),
                ("converged", C.c_int32), ("seconds", C.c_double), ("matvec_seconds", C.c_double),
                ("residual", C.c_double * 64)]

    def as_dict(self):
        return {"iterations": self.iterations, "matvecs": self.matvecs, "restarts": self.restarts,
                "converged": self.converged, "seconds": self.seconds, "matvec_seconds": self.matvec_seconds}


class Stats(C.Structure):
    _fields_ = [("launches", C.c_int64), ("matvecs", C.c_int64), ("stage_launches", C.c_int64 * 5),
                ("stage_ms", C.c_double * 5), ("stage_bytes", C.c_double * 5), ("stage_flops", C.c_double * 5)]

    STAGES = ("k_like", "k_y", "k_z", "k_a", "k_convert")

    def as_dict(self):
        return {"launches": self.launches, "matvecs": self.matvecs,
                "stages": {n: {"launches": self.stage_launches[i], "ms": self.stage_ms[i],
                               "bytes": self.stage_bytes[i], "flops": self.stage_flops[i]}
                           for i, n in enumerate(self.STAGES)}}


class Files(C.Structure):
    _fields_ = [("a", C.c_char_p), ("b", C.c_char_p), ("inter", C.c_char_p), ("like_a", C.c_char_p),
                ("like_b", C.c_char_p), ("T2_a", C.c_int32), ("nmp_a", C.c_int32), ("T2_b", C.c_int32),
                ("nmp_b", C.c_int32), ("xtra", C.c_char), ("J2", C.c_int32), ("parity", C.c_int32),
                ("nshells", C.c_int32), ("nshells_p", C.c_int32), ("shell_parity", _p(C.c_int32))]


class State(C.Structure):
    _fields_ = [("m", C.c_int32), ("V", _p(C.c_double)), ("T", _p(C.c_double)), ("next", _p(C.c_double)),
                ("beta", C.c_double), ("iterations", C.c_int32), ("restarts", C.c_int32)]


class Dop(C.Structure):
    _fields_ = [("nterms", C.c_int32), ("lam2", _p(C.c_int32)), ("parity", _p(C.c_int32)), ("eig", _p(C.c_int32)),
                ("e", _p(C.c_double)), ("shells", _p(C.c_uint8)), ("u", _p(C.c_double))]


class PlanInfo(C.Structure):
    _fields_ = [("y_elems", C.c_int64), ("zbar_elems", C.c_int64), ("zbar_tc_elems", C.c_int64),
                ("y_row_tiles_max", C.c_int32), ("group_sources_max", C.c_int32), ("fused_fp32", C.c_int32),
                ("slab_rows_max", C.c_int32), ("slab_splits_max", C.c_int32), ("slab_nl_max", C.c_int32),
                ("tc_tiles", C.c_int64 * 4), ("tc_chunks_max", C.c_int64), ("fp32_path", C.c_int32),
                ("tc_pieces", C.c_int32)]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_ if f != "tc_tiles"}
        d["tc_tiles"] = [self.tc_tiles[i] for i in range(4)]
        return d


# int fn(void *user, double *y, int64_t n, void *stream): a shard's row exchange (nsx_set_exchange)
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p)

SYMBOLS = {
    "nsx_create": (C.c_int, [_p(Problem), C.c_int, _p(C.c_void_p)]),
    "nsx_create_shard": (C.c_int, [_p(Problem), C.c_int, C.c_int32, C.c_int32, _p(C.c_void_p)]),
    "nsx_load_files_shard": (C.c_int, [_p(Files), C.c_int, C.c_int32, C.c_int32, _p(C.c_void_p)]),
    "nsx_shard_info": (C.c_int, [C.c_void_p, _p(C.c_int32), _p(C.c_int32), _p(C.c_int64), _p(C.c_double)]),
    "nsx_set_exchange": (C.c_int, [C.c_void_p, EXCHANGE_FN, C.c_void_p]),
    "nsx_block_flops": (C.c_int, [C.c_void_p, _p(C.c_double)]),
    "nsx_load_files": (C.c_int, [_p(Files), C.c_int, _p(C.c_void_p)]),
    "nsx_load_files_z": (C.c_int, [_p(Files), C.c_char_p, C.c_int, _p(C.c_void_p)]),
    "nsx_create_z": (C.c_int, [_p(Problem), _p(Dop), C.c_int, _p(C.c_void_p)]),
    "nsx_file_code": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_char_p]),
    "nsx_set_interaction": (C.c_int, [C.c_void_p, _p(C.c_double), C.c_int32, _p(C.c_double), C.c_int64,
                                      _p(C.c_double), C.c_int64]),
    "nsx_dim": (C.c_int64, [C.c_void_p]),
    "nsx_nblocks": (C.c_int32, [C.c_void_p]),
    "nsx_blocks": (C.c_int, [C.c_void_p, _p(C.c_int32), _p(C.c_int64)]),
    "nsx_lcoef": (C.c_int, [C.c_void_p, _p(C.c_uint8)]),
    "nsx_matvec_flops": (C.c_double, [C.c_void_p]),
    "nsx_matvec": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "nsx_matvec_host": (C.c_int, [C.c_void_p, _p(C.c_double), _p(C.c_double), C.c_int32]),
    "nsx_matvec_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "nsx_expectation_matrix": (C.c_int, [C.c_void_p, _p(C.c_double), C.c_int32, C.c_int32, _p(C.c_double)]),
    "nsx_xpct_files": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_int32]),
    "nsx_solve_ex": (C.c_int, [C.c_void_p, _p(Params), _p(State), _p(State), _p(C.c_double), _p(C.c_double),
                               _p(Report)]),
    "nsx_write_state": (C.c_int, [C.c_void_p, C.c_char_p, _p(State), _p(C.c_double), _p(C.c_double), C.c_int32,
                                  C.c_char_p, C.c_int32]),
    "nsx_read_state": (C.c_int, [C.c_void_p, C.c_char_p, _p(State)]),
    "nsx_solve": (C.c_int, [C.c_void_p, _p(Params), _p(C.c_double), _p(C.c_double), _p(Report)]),
    "nsx_batch_solve": (C.c_int, [_p(C.c_void_p), C.c_int32, _p(Params), _p(_p(C.c_double)),
                                  _p(_p(C.c_double)), _p(Report)]),
    "nsx_write_results": (C.c_int, [C.c_void_p, C.c_char_p, _p(C.c_double), _p(C.c_double), C.c_int32, C.c_int32,
                                    C.c_char_p, C.c_int32]),
    "nsx_get_plan_info": (C.c_int, [C.c_void_p, _p(PlanInfo)]),
    "nsx_set_fp32_path": (C.c_int, [C.c_void_p, C.c_int32]),
    "nsx_stats_reset": (C.c_int, [C.c_void_p, C.c_int32]),
    "nsx_get_stats": (C.c_int, [C.c_void_p, _p(Stats)]),
    "nsx_destroy": (None, [C.c_void_p]),
    "nsx_last_error": (C.c_char_p, []),
    "nsx_mlp_create": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.c_int, _p(C.c_void_p)]),
    "nsx_mlp_param_count": (C.c_int64, [C.c_void_p]),
    "nsx_mlp_set_params": (C.c_int, [C.c_void_p, _p(C.c_float), C.c_int64]),
    "nsx_mlp_get_params": (C.c_int, [C.c_void_p, _p(C.c_float), C.c_int64]),
    "nsx_mlp_forward": (C.c_int, [C.c_void_p, _p(C.c_float), C.c_int32, _p(C.c_float)]),
    "nsx_mlp_gradients": (C.c_int, [C.c_void_p, _p(C.c_float), _p(C.c_float), C.c_int32, _p(C.c_float),
                                    _p(C.c_float)]),
    "nsx_mlp_train": (C.c_int, [C.c_void_p, _p(C.c_float), _p(C.c_float), C.c_int32, C.c_int32, C.c_float,
                                _p(C.c_float)]),
    "nsx_mlp_destroy": (None, [C.c_void_p]),
    "nsx_mlp_last_error": (C.c_char_p, []),
}

_lib = None


def load_library(path=LIB_PATH):
    """Load libnsx.so (raises OSError if it is absent: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"libnsx.so not built at {path}: run `python -m nushellx_b200.build`")
    lib = C.CDLL(path)
    for name, (res, args) in SYMBOLS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class NsxError(RuntimeError):
    def __init__(self, rc, msg):
        super().__init__(f"{_ERRNAMES.get(rc, rc)}: {msg}")
        self.rc = rc


def _check(rc):
    if rc != 0:
        raise NsxError(rc, _lib.nsx_last_error().decode(errors="replace"))


def _ptr(a, ctype):
    return a.ctypes.data_as(_p(ctype)) if a is not None and len(a) else None


def _species_struct(keep, S, dens, segs):
    njt = np.zeros(((S.maxJ2 - S.minJ2) // 2 + 1, len(S.parts)), dtype=np.int32)
    for ip in range(len(S.parts)):
        for k in range(njt.shape[0]):
            njt[k, ip] = S.njt(ip, S.minJ2 + 2 * k)
    par = np.array(S.part_parity, dtype=np.int32)
    occ = np.array(S.parts, dtype=np.int16).reshape(len(S.parts), S.norb)   # shell occupations
    arrs = dict(njt=njt.ravel(), par=par, occ=occ.ravel(), keys=dens["keys"], val_off=dens["val_off"],
                vals=np.ascontiguousarray(dens["vals"], dtype=np.float64),
                masks=np.ascontiguousarray(dens["masks"].ravel(), dtype=np.uint32),
                sJ=segs["J2"], snp=segs["np"], snpr=segs["npr"], soff=segs["off"],
                svals=np.ascontiguousarray(segs["vals"], dtype=np.float64))
    keep.append(arrs)
    s = Species()
    s.nspart, s.minJ2, s.maxJ2 = len(S.parts), S.minJ2, S.maxJ2
    s.njt = _ptr(arrs["njt"], C.c_int32)
    s.parity = _ptr(arrs["par"], C.c_int32)
    s.shell_first = S.shell_offset + 1
    s.nshell = S.norb
    s.nkeys = len(arrs["val_off"]) - 1
    s.keys = _ptr(arrs["keys"], C.c_uint8)
    s.val_off = _ptr(arrs["val_off"], C.c_int64)
    s.vals = _ptr(arrs["vals"], C.c_double)
    s.words = dens["words"]
    s.masks = _ptr(arrs["masks"], C.c_uint32)
    s.nseg = len(arrs["sJ"])
    s.seg_J2 = _ptr(arrs["sJ"], C.c_int32)
    s.seg_np = _ptr(arrs["snp"], C.c_int32)
    s.seg_npr = _ptr(arrs["snpr"], C.c_int32)
    s.seg_off = _ptr(arrs["soff"], C.c_int64)
    s.seg_vals = _ptr(arrs["svals"], C.c_double)
    s.occ = _ptr(arrs["occ"], C.c_int16)
    return s


def build_problem_struct(P):
    """nsx_problem for an in-memory generated problem; returns (struct, arrays to keep alive)."""
    from .gen.writer import density_arrays, segment_arrays
    from .gen.pnint import op_order, op_values
    keep = []
    prob = Problem()
    prob.J2, prob.parity = P.J2, P.parity
    prob.a = _species_struct(keep, P.A, density_arrays(P.A, P.rhoA), segment_arrays(P.A, P.segA))
    prob.b = _species_struct(keep, P.B, density_arrays(P.B, P.rhoB), segment_arrays(P.B, P.segB))
    norb = P.space.norb
    okeys = []
    for (o1, o3, o2, o4, lam) in op_order(P.vlam):
        okeys.append(bytes([o1 + 1, o3 + 1, norb + o2 + 1, norb + o4 + 1, lam, 0, 0, 0]))
    ok = np.frombuffer(b"".join(okeys), dtype=np.uint8).copy()
    ov = op_values(P.vlam, op_order(P.vlam))
    keep.append((ok, ov))
    prob.nop = len(ov)
    prob.op_keys = _ptr(ok, C.c_uint8)
    prob.op_vals = _ptr(ov, C.c_double)
    prob.renorm = P.renorm
    return prob, keep


class Solver:
    """One J-scheme problem resident on a GPU."""

    def __init__(self, handle, lib):
        self._h = handle
        self._lib = lib
        self.dim = int(lib.nsx_dim(handle))
        nb = int(lib.nsx_nblocks(handle))
        bb = np.zeros(nb * 4, dtype=np.int32)
        off = np.zeros(nb + 1, dtype=np.int64)
        _check(lib.nsx_blocks(handle, bb.ctypes.data_as(_p(C.c_int32)), off.ctypes.data_as(_p(C.c_int64))))
        self.blocks = bb.reshape(nb, 4)
        self.offsets = off
        m = np.zeros(self.dim, dtype=np.uint8)
        _check(lib.nsx_lcoef(handle, m.ctypes.data_as(_p(C.c_uint8))))
        self.lcoef = m.astype(bool)
        self.flops = float(lib.nsx_matvec_flops(handle))

    # -- construction --------------------------------------------------------------
    @classmethod
    def from_problem(cls, P, device=0, shard=None):
        """From an in-memory generated problem (FP64 operator data, no file rounding).  With
        shard=(rank, world) the handle is rank's output-block shard (nsx_create_shard)."""
        lib = load_library()
        prob, keep = build_problem_struct(P)
        h = C.c_void_p()
        if shard is None:
            _check(lib.nsx_create(C.byref(prob), device, C.byref(h)))
        else:
            _check(lib.nsx_create_shard(C.byref(prob), device, int(shard[0]), int(shard[1]), C.byref(h)))
        return cls(h, lib)

    @classmethod
    def from_problem_z(cls, P, dop_entries, device=0):
        """From an in-memory problem with NuTRLZ's compressed pn interaction (nsx_create_z);
        dop_entries as gen.dop.diop() returns them."""
        lib = load_library()
        prob, keep = build_problem_struct(P)
        rows = [(lam, par, i + 1, e, sh, u) for lam, par, kept in dop_entries
                for i, (e, comps) in enumerate(kept) for (*sh, u) in comps]
        arr = dict(lam2=np.array([r[0] for r in rows], dtype=np.int32),
                   par=np.array([r[1] for r in rows], dtype=np.int32),
                   eig=np.array([r[2] for r in rows], dtype=np.int32),
                   e=np.array([r[3] for r in rows], dtype=np.float64),
                   sh=np.array([r[4] for r in rows], dtype=np.uint8).ravel(),
                   u=np.array([r[5] for r in rows], dtype=np.float64))
        d = Dop()
        d.nterms = len(rows)
        d.lam2, d.parity, d.eig = (_ptr(arr[k], C.c_int32) for k in ("lam2", "par", "eig"))
        d.e, d.u = _ptr(arr["e"], C.c_double), _ptr(arr["u"], C.c_double)
        d.shells = _ptr(arr["sh"], C.c_uint8)
        h = C.c_void_p()
        _check(lib.nsx_create_z(C.byref(prob), C.byref(d), device, C.byref(h)))
        return cls(h, lib)

    @classmethod
    def from_files(cls, manifest, device=0, dop=None, shard=None):
        """From the reference-format files described by a generator manifest (dict or .json path);
        with dop (a .dop path) the pn product uses NuTRLZ's compressed interaction
        (nsx_load_files_z); with shard=(rank, world) the handle is rank's output-block shard
        (nsx_load_files_shard)."""
        lib = load_library()
        if isinstance(manifest, str):
            with open(manifest) as f:
                manifest = json.load(f)
        m = manifest
        sp = np.array(m["shell_parity"], dtype=np.int32)
        f = Files()
        f.a, f.b, f.inter = m["a"].encode(), m["b"].encode(), m["int"].encode()
        f.like_a, f.like_b = m["like_a"].encode(), m["like_b"].encode()
        f.T2_a, f.nmp_a, f.T2_b, f.nmp_b = m["nprot"], -m["nprot"], m["nneut"], m["nneut"]
        f.xtra = b"x"
        f.J2, f.parity = m["J2"], m["parity"]
        f.nshells, f.nshells_p = 2 * m["norb"], m["norb"]
        f.shell_parity = sp.ctypes.data_as(_p(C.c_int32))
        h = C.c_void_p()
        if shard is not None:
            if dop is not None:
                raise ValueError("a shard handle takes the uncompressed interaction")
            _check(lib.nsx_load_files_shard(C.byref(f), device, int(shard[0]), int(shard[1]), C.byref(h)))
        elif dop is None:
            _check(lib.nsx_load_files(C.byref(f), device, C.byref(h)))
        else:
            _check(lib.nsx_load_files_z(C.byref(f), dop.encode(), device, C.byref(h)))
        return cls(h, lib)

    # -- operations -----------------------------------------------------------------
    def matvec_host(self, x, precision=NSX_FP64, out=None):
        """H x with host arrays.  out: the result array (a shard handle without an exchange
        writes its own rows of it and leaves the others)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert x.shape == (self.dim,)
        y = np.empty_like(x) if out is None else out
        assert y.dtype == np.float64 and y.shape == (self.dim,) and y.flags.c_contiguous
        _check(self._lib.nsx_matvec_host(self._h, x.ctypes.data_as(_p(C.c_double)),
                                         y.ctypes.data_as(_p(C.c_double)), precision))
        return y

    def matvec(self, x_ptr, y_ptr, precision=NSX_FP64, stream=None):
        """Device pointers (e.g. torch tensor .data_ptr()); stream is a cudaStream_t integer or None."""
        _check(self._lib.nsx_matvec(self._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr), precision,
                                    C.c_void_p(stream) if stream else None))

    def set_interaction(self, op_vals, a_seg_vals, b_seg_vals):
        """New pn multipole values (order of the creating problem's op keys) and like-particle
        segment values for this handle, without re-planning (nsx_set_interaction)."""
        ov = np.ascontiguousarray(op_vals, dtype=np.float64)
        av = np.ascontiguousarray(a_seg_vals, dtype=np.float64)
        bv = np.ascontiguousarray(b_seg_vals, dtype=np.float64)
        _check(self._lib.nsx_set_interaction(self._h, ov.ctypes.data_as(_p(C.c_double)), len(ov),
                                             av.ctypes.data_as(_p(C.c_double)), len(av),
                                             bv.ctypes.data_as(_p(C.c_double)), len(bv)))

    def matvec_noalloc(self, x_ptr, y_ptr, stream=None):
        """FP64 H.v with the fixed device scratch array (no allocation in the call)."""
        _check(self._lib.nsx_matvec_noalloc(self._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr),
                                            C.c_void_p(stream) if stream else None))

    def expectation_matrix(self, vecs, precision=NSX_FP64):
        """matrixc(i, j) = (H v_i) . v_j for the rows of vecs (NuXpct's matrix; nsx_expectation_matrix)."""
        v = np.ascontiguousarray(vecs, dtype=np.float64)
        assert v.ndim == 2 and v.shape[1] == self.dim
        out = np.zeros((v.shape[0], v.shape[0]), dtype=np.float64, order="F")
        _check(self._lib.nsx_expectation_matrix(self._h, v.ctypes.data_as(_p(C.c_double)), v.shape[0], precision,
                                                out.ctypes.data_as(_p(C.c_double))))
        return out

    def xpct_files(self, xvc_path, out_prefix, precision=NSX_FP64):
        """NuXpct on files: .xvc in, <out_prefix>.ovl / .ovx out (nsx_xpct_files)."""
        _check(self._lib.nsx_xpct_files(self._h, xvc_path.encode(), out_prefix.encode(), precision))

    def solve(self, nev=10, tol=1e-6, precision=NSX_FP64, window=100, keep=0, max_iter=3000, pre_iter=2,
              seed=5, start=None, refine=False, want_vectors=False):
        p = Params()
        p.nev, p.tol, p.precision, p.window, p.keep = nev, tol, precision, window, keep
        p.max_iter, p.pre_iter, p.seed, p.refine = max_iter, pre_iter, seed, int(bool(refine))
        st = None
        if start is not None:
            st = np.ascontiguousarray(start, dtype=np.float64)
            p.start = st.ctypes.data_as(_p(C.c_double))
        ev = np.zeros(nev)
        vecs = np.zeros((nev, self.dim)) if want_vectors else None
        rep = Report()
        _check(self._lib.nsx_solve(self._h, C.byref(p), ev.ctypes.data_as(_p(C.c_double)),
                                   vecs.ctypes.data_as(_p(C.c_double)) if vecs is not None else None,
                                   C.byref(rep)))
        out = rep.as_dict()
        out["residual"] = [rep.residual[i] for i in range(min(nev, 64))]
        return ev, vecs, out

    def solve_state(self, nev=10, tol=1e-6, precision=NSX_FP64, window=100, keep=0, max_iter=3000, pre_iter=2,
                    seed=5, start=None, refine=False, resume=None):
        """nsx_solve_ex: a solve that returns its thick-restart state (dict V, T, next, beta,
        iterations, restarts) and can resume from one.  Returns (evals, vecs, report, state)."""
        p = Params()
        p.nev, p.tol, p.precision, p.window, p.keep = nev, tol, precision, window, keep
        p.max_iter, p.pre_iter, p.seed, p.refine = max_iter, pre_iter, seed, int(bool(refine))
        st = None
        if start is not None:
            st = np.ascontiguousarray(start, dtype=np.float64)
            p.start = st.ctypes.data_as(_p(C.c_double))
        keep_alive = []
        rs = None
        if resume is not None:
            V = np.ascontiguousarray(resume["V"], dtype=np.float64)
            T = np.asfortranarray(resume["T"], dtype=np.float64)
            nx = np.ascontiguousarray(resume["next"], dtype=np.float64)
            keep_alive += [V, T, nx]
            rs = State(V.shape[0], V.ctypes.data_as(_p(C.c_double)), T.ctypes.data_as(_p(C.c_double)),
                       nx.ctypes.data_as(_p(C.c_double)), float(resume["beta"]), int(resume.get("iterations", 0)),
                       int(resume.get("restarts", 0)))
        cap = min(window, 112) + 1
        Vo = np.zeros((cap, self.dim))
        To = np.zeros(cap * cap)
        No = np.zeros(self.dim)
        so = State(cap, Vo.ctypes.data_as(_p(C.c_double)), To.ctypes.data_as(_p(C.c_double)),
                   No.ctypes.data_as(_p(C.c_double)), 0.0, 0, 0)
        ev = np.zeros(nev)
        vecs = np.zeros((nev, self.dim))
        rep = Report()
        _check(self._lib.nsx_solve_ex(self._h, C.byref(p), C.byref(rs) if rs is not None else None, C.byref(so),
                                      ev.ctypes.data_as(_p(C.c_double)), vecs.ctypes.data_as(_p(C.c_double)),
                                      C.byref(rep)))
        m = so.m
        state = {"V": Vo[:m].copy(), "T": To[:m * m].reshape(m, m, order="F").copy(), "next": No, "beta": so.beta,
                 "iterations": so.iterations, "restarts": so.restarts}
        out = rep.as_dict()
        out["residual"] = [rep.residual[i] for i in range(min(nev, 64))]
        return ev, vecs, out, state

    def write_state(self, prefix, state, evals, vecs=None, intfile="", T2=0):
        """The reference's TRL files for a state (nsx_write_state): .abz/.trl, .lev, .xvc."""
        V = np.ascontiguousarray(state["V"], dtype=np.float64)
        T = np.asfortranarray(state["T"], dtype=np.float64)
        nx = np.ascontiguousarray(state["next"], dtype=np.float64)
        st = State(V.shape[0], V.ctypes.data_as(_p(C.c_double)), T.ctypes.data_as(_p(C.c_double)),
                   nx.ctypes.data_as(_p(C.c_double)), float(state["beta"]), int(state["iterations"]),
                   int(state["restarts"]))
        ev = np.ascontiguousarray(evals, dtype=np.float64)
        vv = np.ascontiguousarray(vecs, dtype=np.float64) if vecs is not None else None
        _check(self._lib.nsx_write_state(self._h, prefix.encode(), C.byref(st), ev.ctypes.data_as(_p(C.c_double)),
                                         vv.ctypes.data_as(_p(C.c_double)) if vv is not None else None, len(ev),
                                         intfile.encode(), int(T2)))

    def read_state(self, prefix, cap=113):
        """A state written by write_state (nsx_read_state)."""
        Vo = np.zeros((cap, self.dim))
        To = np.zeros(cap * cap)
        No = np.zeros(self.dim)
        so = State(cap, Vo.ctypes.data_as(_p(C.c_double)), To.ctypes.data_as(_p(C.c_double)),
                   No.ctypes.data_as(_p(C.c_double)), 0.0, 0, 0)
        _check(self._lib.nsx_read_state(self._h, prefix.encode(), C.byref(so)))
        m = so.m
        return {"V": Vo[:m].copy(), "T": To[:m * m].reshape(m, m, order="F").copy(), "next": No, "beta": so.beta,
                "iterations": so.iterations, "restarts": so.restarts}

    def write_results(self, prefix, evals, vecs, iterations=0, intfile="", T2=0):
        """The reference's .abz / .trl / .lev files for these eigenpairs (nsx_write_results)."""
        ev = np.ascontiguousarray(evals, dtype=np.float64)
        vv = np.ascontiguousarray(vecs, dtype=np.float64)
        assert vv.shape == (len(ev), self.dim)
        _check(self._lib.nsx_write_results(self._h, prefix.encode(), ev.ctypes.data_as(_p(C.c_double)),
                                           vv.ctypes.data_as(_p(C.c_double)), len(ev), int(iterations),
                                           intfile.encode(), int(T2)))

    @staticmethod
    def batch_solve(solvers, nev=10, tol=1e-6, precision=NSX_FP64, window=100, max_iter=3000, refine=False,
                    want_vectors=False):
        """Independent solves of distinct solvers at once (nsx_batch_solve); returns a list of
        (eigenvalues, eigenvectors or None, report) in the order of `solvers`."""
        lib = load_library()
        n = len(solvers)
        hs = (C.c_void_p * n)(*[s._h for s in solvers])
        ps = (Params * n)()
        for p in ps:
            p.nev, p.tol, p.precision, p.window, p.keep = nev, tol, precision, window, 0
            p.max_iter, p.pre_iter, p.seed, p.refine = max_iter, 2, 5, int(bool(refine))
        evs = [np.zeros(nev) for _ in range(n)]
        vecs = [np.zeros((nev, s.dim)) for s in solvers] if want_vectors else None
        ev_ptrs = (_p(C.c_double) * n)(*[e.ctypes.data_as(_p(C.c_double)) for e in evs])
        vec_ptrs = (_p(C.c_double) * n)(*[v.ctypes.data_as(_p(C.c_double)) for v in vecs]) if vecs else None
        reps = (Report * n)()
        _check(lib.nsx_batch_solve(hs, n, ps, ev_ptrs, vec_ptrs, reps))
        out = []
        for i in range(n):
            r = reps[i].as_dict()
            r["residual"] = [reps[i].residual[k] for k in range(min(nev, 64))]
            out.append((evs[i], vecs[i] if vecs else None, r))
        return out

    def shard_info(self):
        """{"rank", "world", "rows": first row of every rank (world + 1 entries), "est_flops"}."""
        rank, world = C.c_int32(), C.c_int32()
        _check(self._lib.nsx_shard_info(self._h, C.byref(rank), C.byref(world), None, None))
        rows = np.zeros(world.value + 1, dtype=np.int64)
        fl = np.zeros(world.value, dtype=np.float64)
        _check(self._lib.nsx_shard_info(self._h, None, None, _ptr(rows, C.c_int64), _ptr(fl, C.c_double)))
        return {"rank": rank.value, "world": world.value, "rows": rows, "est_flops": fl}

    def block_flops(self):
        """The flops of every output block's rows (what the shard split balances)."""
        out = np.zeros(len(self.blocks), dtype=np.float64)
        _check(self._lib.nsx_block_flops(self._h, _ptr(out, C.c_double)))
        return out

    def set_exchange(self, fn):
        """Every product of this shard handle ends with fn(y_ptr, n, stream_ptr), which must fill
        the other ranks' rows of the device vector y (an all-gather) in the order of `stream`.
        fn=None removes it.  An exception inside fn fails the product (NSX_E_CUDA) and is
        kept in self.exchange_error."""
        if fn is None:
            self._exchange = None
            _check(self._lib.nsx_set_exchange(self._h, EXCHANGE_FN(), None))
            return
        self.exchange_error = None

        def cb(user, y, n, stream):
            try:
                fn(int(y or 0), int(n), int(stream or 0))
                return 0
            except BaseException as e:   # never let an exception cross the C frames
                self.exchange_error = e
                return 1

        self._exchange = EXCHANGE_FN(cb)   # kept alive as long as the handle may call it
        _check(self._lib.nsx_set_exchange(self._h, self._exchange, None))

    def stats_reset(self, timing=False):
        _check(self._lib.nsx_stats_reset(self._h, 1 if timing else 0))

    def set_fp32_path(self, path):
        """NSX_FP32_AUTO (0), NSX_FP32_FUSED (1), NSX_FP32_TC (2) or NSX_FP32_SIMT (3)."""
        _check(self._lib.nsx_set_fp32_path(self._h, int(path)))

    def plan_info(self):
        """Which H.v kernel paths this handle's products take (nsx_get_plan_info)."""
        pi = PlanInfo()
        _check(self._lib.nsx_get_plan_info(self._h, C.byref(pi)))
        return pi.as_dict()

    def stats(self):
        st = Stats()
        _check(self._lib.nsx_get_stats(self._h, C.byref(st)))
        return st.as_dict()

    def close(self):
        if self._h:
            self._lib.nsx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _mcheck(rc):
    if rc != 0:
        raise NsxError(rc, _lib.nsx_mlp_last_error().decode(errors="replace"))


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class Network:
    """The learned start vector's MLP on a GPU (nsx_mlp_*): n_in -> width -> width -> n_out."""

    def __init__(self, n_in, width, n_out, seed=1, device=0):
        self._lib = load_library()
        self._h = C.c_void_p()
        _mcheck(self._lib.nsx_mlp_create(n_in, width, n_out, seed, device, C.byref(self._h)))
        self.n_in, self.width, self.n_out = n_in, width, n_out
        self.nparams = int(self._lib.nsx_mlp_param_count(self._h))

    @property
    def params(self):
        p = np.zeros(self.nparams, dtype=np.float32)
        _mcheck(self._lib.nsx_mlp_get_params(self._h, p.ctypes.data_as(_p(C.c_float)), self.nparams))
        return p

    @params.setter
    def params(self, p):
        p = _f32(p)
        _mcheck(self._lib.nsx_mlp_set_params(self._h, p.ctypes.data_as(_p(C.c_float)), len(p)))

    def forward(self, x):
        x = _f32(x).reshape(-1, self.n_in)
        y = np.zeros((len(x), self.n_out), dtype=np.float32)
        _mcheck(self._lib.nsx_mlp_forward(self._h, x.ctypes.data_as(_p(C.c_float)), len(x),
                                          y.ctypes.data_as(_p(C.c_float))))
        return y

    def gradients(self, x, t):
        x, t = _f32(x).reshape(-1, self.n_in), _f32(t).reshape(-1, self.n_out)
        loss = C.c_float()
        g = np.zeros(self.nparams, dtype=np.float32)
        _mcheck(self._lib.nsx_mlp_gradients(self._h, x.ctypes.data_as(_p(C.c_float)),
                                            t.ctypes.data_as(_p(C.c_float)), len(x), C.byref(loss),
                                            g.ctypes.data_as(_p(C.c_float))))
        return float(loss.value), g

    def train(self, x, t, steps, lr):
        x, t = _f32(x).reshape(-1, self.n_in), _f32(t).reshape(-1, self.n_out)
        loss = C.c_float()
        _mcheck(self._lib.nsx_mlp_train(self._h, x.ctypes.data_as(_p(C.c_float)), t.ctypes.data_as(_p(C.c_float)),
                                        len(x), steps, lr, C.byref(loss)))
        return float(loss.value)

    def close(self):
        if self._h:
            self._lib.nsx_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
