"""Python mirror of the bipp API (python/pybipp.cpp:285-493) over the C ABI.

Same names, argument meaning and error behaviour as the reference's pybind module
``bipp.pybipp`` for the Bluebild path: ``Context``, ``eigh``, ``eigh_gram``,
``NufftSynthesisOptions``, ``Partition``, ``image_synthesis``; plus the internal
entry points the reference does not bind (``gram_matrix``, ``virtual_vis``,
``nuft_sum``, ``domain_partition_grid``, the collect/get ``NufftSynthesis``) and
the batched ``Pipeline``. Every numeric call runs on the GPU through
libbipp_b200.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from typing import Dict, Mapping, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import BippError, EigensolverError, InvalidParameterError, GPUError, check  # noqa: F401

_PU = {"AUTO": _lib.BIPP_PU_AUTO, "CPU": _lib.BIPP_PU_CPU, "GPU": _lib.BIPP_PU_GPU}


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class _CompileConfig:
    """pybipp's ``config`` (python/pybipp.cpp:295-302): what the library was built with.
    CUDA only; multi-rank runs use torch.distributed, not MPI."""

    cuda, rocm, umpire, omp, mpi = True, False, False, False, False


config = _CompileConfig()


class communicator:
    """pybipp's ``communicator`` (python/pybipp.cpp:304-308, include/bipp/communicator.hpp:22-89):
    ``communicator.world()`` is the job of one process per GPU, read from the RANK and
    WORLD_SIZE variables that torch.distributed launchers set (the reference reads
    MPI_COMM_WORLD); ``communicator.local()`` is this process alone. The transport of
    the image reduction is torch.distributed (NCCL on GPUs), which must be initialised
    when size > 1."""

    def __init__(self, rank: int = 0, size: int = 1):
        if size < 1 or not 0 <= rank < size:
            raise InvalidParameterError(3, f"invalid communicator rank {rank} of {size}")
        self._rank, self._size = int(rank), int(size)

    @staticmethod
    def world() -> "communicator":
        return communicator(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")))

    @staticmethod
    def local() -> "communicator":
        return communicator(0, 1)

    @property
    def rank(self) -> int:
        return self._rank

    @property
    def size(self) -> int:
        return self._size


class Context:
    """Context(pu) or Context(pu, comm) with pu in {"AUTO", "GPU"} (include/bipp/context.hpp:25-66,
    python/pybipp.cpp:310-315). "CPU" raises InvalidParameterError: this library has no
    CPU processing unit. With a communicator, the GPU is rank % device count as in the
    reference (src/context_internal.cpp:59-66) unless `device` is given, and
    image_synthesis splits the samples over the ranks."""

    def __init__(self, pu: str = "AUTO", comm: Optional[communicator] = None, device: Optional[int] = None):
        self._lib = _lib.load()
        self.communicator = comm if comm is not None else communicator.local()
        h = C.c_void_p()
        code = _PU[pu.upper()] if isinstance(pu, str) else int(pu)
        if device is None and comm is not None and self.communicator.size > 1:
            import torch

            device = pick_device(self.communicator, torch.cuda.device_count())
        # the GPU of this context (None: the CUDA device current at creation); collectives
        # over this context's images run on it
        self.device = device
        if device is None:
            check(self._lib.bipp_ctx_create(code, C.byref(h)))
        else:
            check(self._lib.bipp_ctx_create_on_device(code, int(device), C.byref(h)))
        self.handle = h

    @property
    def processing_unit(self) -> str:
        """"AUTO", "CPU" or "GPU" (a read-only property, as pybipp's)."""
        pu = C.c_int()
        check(self._lib.bipp_ctx_processing_unit(self.handle, C.byref(pu)))
        return {0: "AUTO", 1: "CPU", 2: "GPU"}[pu.value]

    def stream(self) -> int:
        s = C.c_void_p()
        check(self._lib.bipp_ctx_stream(self.handle, C.byref(s)))
        return s.value or 0

    def close(self):
        if getattr(self, "handle", None):
            self._lib.bipp_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None
_default_lock = threading.Lock()


def default_context() -> Context:
    """Process-wide context used by the context-free entry points (eigh, eigh_gram)."""
    global _default_ctx
    with _default_lock:
        if _default_ctx is None:
            _default_ctx = Context("AUTO")
        return _default_ctx


def kernel_launch_count() -> int:
    """Kernels this library has launched in this process so far (cuFFT's excluded)."""
    return int(_lib.load().bipp_kernel_launch_count())


def _prec(wl, *arrays):
    dbl = isinstance(wl, (np.float64, float)) and not isinstance(wl, np.float32)
    for a in arrays:
        if a is not None and np.asarray(a).dtype in (np.complex64, np.float32):
            dbl = False
    return dbl


# --- eigensolvers ---------------------------------------------------------------------

def eigh_gram(wl, s, w, xyz, ctx: Optional[Context] = None, precision: Optional[str] = None):
    """(v, d, scale) = eigh_gram(wl, s, w, xyz); python/pybipp.cpp:254-275, 462-477.
    Single precision when the arrays are complex64/float32, double otherwise."""
    ctx = ctx or default_context()
    dbl = (precision == "double") if precision else _prec(wl, s, w, xyz)
    rt, ct = (np.float64, np.complex128) if dbl else (np.float32, np.complex64)
    s = np.asfortranarray(s, dtype=ct)
    w = np.asfortranarray(w, dtype=ct)
    xyz = np.asfortranarray(xyz, dtype=rt)
    n_ant, n_beam = w.shape
    if s.shape != (n_beam, n_beam) or xyz.shape != (n_ant, 3):
        raise InvalidParameterError(3, "inconsistent array shapes")
    d = np.zeros(n_beam, dtype=rt)
    v = np.zeros((n_ant, n_beam), dtype=ct, order="F")
    nred = C.c_size_t()
    scale = (C.c_double if dbl else C.c_float)()
    fn = ctx._lib.bipp_eigh_gram_d if dbl else ctx._lib.bipp_eigh_gram_s
    check(fn(ctx.handle, rt(wl), n_ant, n_beam, _ptr(s), n_beam, _ptr(w), n_ant, _ptr(xyz), n_ant, _ptr(d),
             _ptr(v), n_ant, C.byref(nred), C.byref(scale)))
    return v, d, scale.value


def eigh_gram_full(wl, s, w, xyz, ctx: Optional[Context] = None, precision: Optional[str] = None):
    """As eigh_gram, also returning nBeamReduced: (v, d, nReduced, scale)."""
    ctx = ctx or default_context()
    dbl = (precision == "double") if precision else _prec(wl, s, w, xyz)
    rt, ct = (np.float64, np.complex128) if dbl else (np.float32, np.complex64)
    s = np.asfortranarray(s, dtype=ct)
    w = np.asfortranarray(w, dtype=ct)
    xyz = np.asfortranarray(xyz, dtype=rt)
    n_ant, n_beam = w.shape
    d = np.zeros(n_beam, dtype=rt)
    v = np.zeros((n_ant, n_beam), dtype=ct, order="F")
    nred = C.c_size_t()
    scale = (C.c_double if dbl else C.c_float)()
    fn = ctx._lib.bipp_eigh_gram_d if dbl else ctx._lib.bipp_eigh_gram_s
    check(fn(ctx.handle, rt(wl), n_ant, n_beam, _ptr(s), n_beam, _ptr(w), n_ant, _ptr(xyz), n_ant, _ptr(d),
             _ptr(v), n_ant, C.byref(nred), C.byref(scale)))
    return v, d, nred.value, scale.value


def eigh(wl, s, w, ctx: Optional[Context] = None, precision: Optional[str] = None, full: bool = False):
    """(v, d, scale) = eigh(wl, s, w); python/pybipp.cpp:234-252, 478-492."""
    ctx = ctx or default_context()
    dbl = (precision == "double") if precision else _prec(wl, s, w)
    rt, ct = (np.float64, np.complex128) if dbl else (np.float32, np.complex64)
    s = np.asfortranarray(s, dtype=ct)
    w = np.asfortranarray(w, dtype=ct)
    n_ant, n_beam = w.shape
    d = np.zeros(n_beam, dtype=rt)
    v = np.zeros((n_ant, n_beam), dtype=ct, order="F")
    nred = C.c_size_t()
    scale = (C.c_double if dbl else C.c_float)()
    fn = ctx._lib.bipp_eigh_d if dbl else ctx._lib.bipp_eigh_s
    check(fn(ctx.handle, rt(wl), n_ant, n_beam, _ptr(s), n_beam, _ptr(w), n_ant, _ptr(d), _ptr(v), n_ant,
             C.byref(nred), C.byref(scale)))
    return (v, d, nred.value, scale.value) if full else (v, d, scale.value)


def eigh_gram_batched(wl, s, xyz, ctx: Optional[Context] = None, precision: str = "single"):
    """Batched eigh_gram with W = I over steps: wl [B], s [B, N, N] (s[b] is the step's
    matrix; its lower triangle in column-major order is used), xyz [B, N, 3]. Single
    precision (complex64, bipp_eigh_gram_batched_s) or "double" (complex128,
    bipp_eigh_gram_batched_d). Returns (v [B, N, N] (v[b][:, c] eigenvector c), d [B, N],
    nReduced [B], scale [B])."""
    ctx = ctx or default_context()
    dbl = precision == "double"
    rt, ct = (np.float64, np.complex128) if dbl else (np.float32, np.complex64)
    wl = np.ascontiguousarray(wl, dtype=rt)
    s = np.asarray(s, dtype=ct)
    B, N = s.shape[0], s.shape[1]
    # column-major per matrix: store transposed so that memory order matches F layout
    sF = np.ascontiguousarray(np.transpose(s, (0, 2, 1)))
    xyzF = np.ascontiguousarray(np.transpose(np.asarray(xyz, dtype=rt), (0, 2, 1)))
    d = np.zeros((B, N), dtype=rt)
    vF = np.zeros((B, N, N), dtype=ct)
    nred = np.zeros(B, dtype=np.uint64)
    scale = np.zeros(B, dtype=rt)
    fn = ctx._lib.bipp_eigh_gram_batched_d if dbl else ctx._lib.bipp_eigh_gram_batched_s
    check(fn(ctx.handle, B, N, _ptr(wl), _ptr(sF), _ptr(xyzF), _ptr(d), _ptr(vF), _ptr(nred), _ptr(scale)))
    v = np.transpose(vF, (0, 2, 1))
    return v, d, nred.astype(np.int64), scale


def gram_matrix(xyz, w, wl, ctx: Optional[Context] = None):
    """G = W^H sinc(2|p_i - p_j|/wl) W (src/host/gram_matrix.cpp:29-64); the Python
    pipeline expects pybipp.gram_matrix(ctx, xyz, w, wl) (python/bipp/gram.py:98-103)."""
    ctx = ctx or default_context()
    dbl = _prec(wl, w, xyz)
    rt, ct = (np.float64, np.complex128) if dbl else (np.float32, np.complex64)
    w = np.asfortranarray(w, dtype=ct)
    xyz = np.asfortranarray(xyz, dtype=rt)
    n_ant, n_beam = w.shape
    g = np.zeros((n_beam, n_beam), dtype=ct, order="F")
    fn = ctx._lib.bipp_gram_matrix_d if dbl else ctx._lib.bipp_gram_matrix_s
    check(fn(ctx.handle, n_ant, n_beam, _ptr(w), n_ant, _ptr(xyz), n_ant, rt(wl), _ptr(g), n_beam))
    return g


def virtual_vis(scale, d, v, ctx: Optional[Context] = None):
    """VV = V_k diag(scale d_k) V_k^H over non-zero d (src/host/virtual_vis.cpp:19-73),
    returned as the nAntenna x nAntenna matrix."""
    ctx = ctx or default_context()
    v = np.asarray(v)
    dbl = v.dtype == np.complex128
    rt, ct = (np.float64, np.complex128) if dbl else (np.float32, np.complex64)
    v = np.asfortranarray(v, dtype=ct)
    d = np.ascontiguousarray(d, dtype=rt)
    n_ant, n_beam = v.shape
    vv = np.zeros((n_ant, n_ant), dtype=ct, order="F")
    fn = ctx._lib.bipp_virtual_vis_d if dbl else ctx._lib.bipp_virtual_vis_s
    check(fn(ctx.handle, rt(scale), n_ant, n_beam, _ptr(d), _ptr(v), n_ant, _ptr(vv)))
    return vv


def nuft_sum(alpha, values, u, v, w, x, y, z, out=None, ctx: Optional[Context] = None):
    """out[p] += Re sum_k values_k exp(i alpha (x_p u_k + y_p v_k + z_p w_k))
    (src/host/kernels/nuft_sum.cpp:9-31)."""
    ctx = ctx or default_context()
    values = np.asarray(values)
    dbl = values.dtype == np.complex128
    rt, ct = (np.float64, np.complex128) if dbl else (np.float32, np.complex64)
    values = np.ascontiguousarray(values, dtype=ct)
    u, v, w, x, y, z = (np.ascontiguousarray(a, dtype=rt) for a in (u, v, w, x, y, z))
    if out is None:
        out = np.zeros(x.shape[0], dtype=rt)
    fn = ctx._lib.bipp_nuft_sum_d if dbl else ctx._lib.bipp_nuft_sum_s
    check(fn(ctx.handle, rt(alpha), values.shape[0], _ptr(values), _ptr(u), _ptr(v), _ptr(w), x.shape[0], _ptr(x),
             _ptr(y), _ptr(z), _ptr(out)))
    return out


def domain_partition_grid(dims, x, y, z, ctx: Optional[Context] = None):
    """(permut, group_begin, group_size) of DomainPartition::grid
    (src/host/domain_partition.hpp:35-101); permut[i] = sorted position of point i."""
    ctx = ctx or default_context()
    x = np.asarray(x)
    dbl = x.dtype == np.float64
    rt = np.float64 if dbl else np.float32
    x, y, z = (np.ascontiguousarray(a, dtype=rt) for a in (x, y, z))
    dims = np.ascontiguousarray(dims, dtype=np.uint64)
    ng = int(np.prod(dims))
    n = x.shape[0]
    permut = np.zeros(n, dtype=np.uint64)
    gb = np.zeros(max(ng, 1), dtype=np.uint64)
    gs = np.zeros(max(ng, 1), dtype=np.uint64)
    fn = ctx._lib.bipp_domain_partition_grid_d if dbl else ctx._lib.bipp_domain_partition_grid_s
    check(fn(ctx.handle, _ptr(dims), n, _ptr(x), _ptr(y), _ptr(z), _ptr(permut), _ptr(gb), _ptr(gs)))
    if ng <= 1:
        return permut, gb[:1], gs[:1]
    return permut, gb, gs


# --- options -----------------------------------------------------------------------------

class Partition:
    """Partition.auto() / Partition.none() / Partition.grid([u, v, w])
    (include/bipp/image_synthesis.hpp:23-53)."""

    def __init__(self, method: str = "auto", dims: Sequence[int] = (1, 1, 1)):
        self.method = method
        self.dims = tuple(int(d) for d in dims)

    @staticmethod
    def auto():
        return Partition("auto")

    @staticmethod
    def none():
        return Partition("none")

    @staticmethod
    def grid(dims):
        return Partition("grid", dims)


class NufftSynthesisOptions:
    """include/bipp/image_synthesis.hpp:55-148 (apply_scaling is accepted; the scale
    is always applied, as in the reference, src/nufft_synthesis.cpp:138,160)."""

    def __init__(self):
        self.precision = "single"
        self.tolerance = 0.001
        self.sample_batch_size = None
        self.local_uvw_partition = Partition.auto()
        self.normalize_image = True
        self.apply_scaling = True

    def set_tolerance(self, tol):
        self.tolerance = float(tol)
        return self

    def set_sample_batch_size(self, size):
        self.sample_batch_size = size
        return self

    def set_local_uvw_partition(self, p: Partition):
        self.local_uvw_partition = p
        return self

    def set_normalize_image(self, normalize: bool):
        self.normalize_image = bool(normalize)
        return self

    def set_apply_scaling(self, apply: bool):
        self.apply_scaling = bool(apply)
        return self

    def set_precision(self, prec: str):
        if prec not in ("single", "double"):
            raise InvalidParameterError(3, f"unknown precision {prec}")
        self.precision = prec
        return self

    def _c(self) -> _lib.NufftOptions:
        o = _lib.NufftOptions()
        o.precision = _lib.BIPP_PRECISION_DOUBLE if self.precision == "double" else _lib.BIPP_PRECISION_SINGLE
        o.tolerance = self.tolerance
        o.sampleBatchSize = int(self.sample_batch_size or 0)
        o.partitionMethod = {"auto": 0, "none": 1, "grid": 2}[self.local_uvw_partition.method]
        for i in range(3):
            o.partitionGrid[i] = self.local_uvw_partition.dims[i]
        o.normalizeImage = 1 if self.normalize_image else 0
        o.applyScaling = 1 if self.apply_scaling else 0
        return o


# --- collect / get NUFFT ------------------------------------------------------------------

class NufftSynthesis:
    """Collect/get object mirroring NUFFTInterface::add / get_image
    (src/nufft_interface.hpp:13-21): add(uvw [nBaselines, 3] scaled by 2 pi/wl,
    values [nBaselines, nImages]) and get_image(i) -> [nPixel] float32."""

    def __init__(self, ctx: Context, opt: NufftSynthesisOptions, lmn, n_images: int, n_baselines: int):
        self.ctx = ctx
        lmn = np.asfortranarray(lmn, dtype=np.float32)
        self.n_pixel = lmn.shape[0]
        self.n_images = int(n_images)
        self.n_baselines = int(n_baselines)
        h = C.c_void_p()
        o = opt._c()
        check(ctx._lib.bipp_nufft_create(ctx.handle, C.byref(o), self.n_pixel, _ptr(lmn), self.n_pixel,
                                         self.n_images, self.n_baselines, C.byref(h)))
        self.handle = h

    def add(self, uvw, values):
        uvw = np.asarray(uvw)
        if uvw.dtype == np.float64:
            uvw = np.asfortranarray(uvw)
            values = np.asfortranarray(values, dtype=np.complex128)
            check(self.ctx._lib.bipp_nufft_add_d(self.handle, _ptr(uvw), uvw.shape[0], _ptr(values), values.shape[0]))
        else:
            uvw = np.asfortranarray(uvw, dtype=np.float32)
            values = np.asfortranarray(values, dtype=np.complex64)
            check(self.ctx._lib.bipp_nufft_add_s(self.handle, _ptr(uvw), uvw.shape[0], _ptr(values), values.shape[0]))

    def get_image(self, idx: int):
        img = np.zeros(self.n_pixel, dtype=np.float32)
        check(self.ctx._lib.bipp_nufft_get_image(self.handle, int(idx), _ptr(img)))
        return img

    def close(self):
        if getattr(self, "handle", None):
            self.ctx._lib.bipp_nufft_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --- dataset-driven image synthesis --------------------------------------------------------

class InMemoryDataset:
    """In-memory Dataset (include/bipp/dataset.hpp:14-41): per sample eigenvectors
    (nAnt x nBeam complex), eigenvalues (nBeam), uvw (nAnt^2 x 3, metres), wl, scale."""

    def __init__(self, n_antenna, n_beam, description=""):
        self.n_antenna, self.n_beam, self.description = n_antenna, n_beam, description
        self.samples = []

    def write(self, time_stamp, wl, scale, v, d, uvw):
        self.samples.append(dict(t=float(time_stamp), wl=float(wl), scale=float(scale),
                                 v=np.asfortranarray(v, dtype=np.complex64), d=np.asarray(d, dtype=np.float32),
                                 uvw=np.asfortranarray(uvw, dtype=np.float32)))

    def num_samples(self):
        return len(self.samples)

    def num_antenna(self):
        return self.n_antenna

    def num_beam(self):
        return self.n_beam

    def eig_vec(self, i):
        return self.samples[i]["v"]

    def eig_val(self, i):
        return self.samples[i]["d"]

    def uvw(self, i):
        return self.samples[i]["uvw"]

    def wl(self, i):
        return self.samples[i]["wl"]

    def scale(self, i):
        return self.samples[i]["scale"]


def image_synthesis(ctx: Context, opt: NufftSynthesisOptions, dataset, selection: Mapping[str, Mapping[int, Sequence[float]]],
                    image_prop, image_file_name: Optional[str] = None) -> Dict[str, np.ndarray]:
    """image_synthesis(ctx, opt, dataset, selection, image_prop, image_file_name)
    (python/pybipp.cpp:176-196, include/bipp/image_synthesis.hpp:160-163).

    selection: {tag: {sample_id: scaled eigenvalues [nBeam]}}; image_prop: an object
    with pixel_lmn() -> [nPixel, 3] or the lmn array itself. Returns {tag: image}; if
    image_file_name is given the images are also saved there with numpy.savez (the
    reference's HDF5 image file format is not implemented).

    With a context of several ranks (Context(pu, communicator.world())) every rank
    images its contiguous block of the sorted sample ids, the images are summed into
    rank 0 over torch.distributed and normalised there by the total sample count
    (src/image_synthesis.cpp:71-80, 140-163); rank 0 returns the images, the other
    ranks an empty dict."""
    tags = _check_tags(selection)
    lmn = image_prop.pixel_lmn() if hasattr(image_prop, "pixel_lmn") else image_prop
    comm = getattr(ctx, "communicator", None) or communicator.local()
    if comm.size == 1:
        images = _synthesize(ctx, opt, dataset, selection, tags, lmn, opt.normalize_image)
    else:
        local, n_total = split_selection(selection, dataset.num_samples(), comm.rank, comm.size)
        if len(local[tags[0]]):
            images = _synthesize(ctx, opt, dataset, local, tags, lmn, False)
        else:
            images = np.zeros((len(tags), np.asarray(lmn).shape[0]), dtype=np.float32)
        images = _reduce_images_to_root(images, getattr(ctx, "device", None))
        if comm.rank != 0:
            return {}
        if opt.normalize_image:
            images *= np.float32(1.0) / np.float32(n_total)
    out = {tag: images[i] for i, tag in enumerate(tags)}
    if image_file_name:
        np.savez(image_file_name, **out)
    return out


def _check_tags(selection) -> list:
    for tag in selection:
        if "/" in tag:
            raise InvalidParameterError(3, "Selection name must not contain '/'")
        if "." in tag:
            raise InvalidParameterError(3, "Selection name must not contain '.'")
        if " " in tag:
            raise InvalidParameterError(3, "Selection name must not contain spaces")
    tags = list(selection.keys())
    if not tags:
        raise InvalidParameterError(3, "Empty selection")
    return tags


def split_selection(selection, n_dataset: int, rank: int, size: int):
    """The block of `rank` among `size` ranks: per tag, the samples at positions
    [rank * ceil(n / size), ...) of the id-sorted selection, after the reference's checks
    over the whole selection (src/image_synthesis.cpp:44-105: no duplicate ids, ids below
    the dataset's sample count, the same ids for every image). Returns ({tag: {id: ev}},
    total sample count)."""
    from .distributed import sample_split

    tags = list(selection.keys())
    if not tags:
        raise InvalidParameterError(3, "Empty selection")
    order = {}
    for tag in tags:
        ids = sorted(int(i) for i in selection[tag].keys())
        if not ids:
            raise InvalidParameterError(3, "Empty selection")
        if len(set(ids)) != len(ids):
            raise InvalidParameterError(3, "Selection sample id duplicate")
        if ids[-1] >= n_dataset:
            raise InvalidParameterError(3, "Selection sample id exceeds number of dataset samples")
        order[tag] = ids
    n_total = len(order[tags[0]])
    for tag in tags:
        if order[tag] != order[tags[0]]:
            raise InvalidParameterError(3, "Selection must contain the same sample ids for all images.")
    begin, count = sample_split(n_total, rank, size)
    keys = {tag: {int(k): k for k in selection[tag].keys()} for tag in tags}
    local = {tag: {i: selection[tag][keys[tag][i]] for i in order[tag][begin:begin + count]} for tag in tags}
    return local, n_total


def pick_device(comm: communicator, n_devices: int) -> Optional[int]:
    """GPU of a rank under a multi-rank communicator: rank % device count, as the
    reference (src/context_internal.cpp:59-66); None without devices."""
    return comm.rank % n_devices if n_devices else None


def _reduce_images_to_root(images: np.ndarray, device: Optional[int] = None) -> np.ndarray:
    """Sum the [nImages, nPixel] float images of all ranks into rank 0 (NCCL on GPUs, on
    the context's device)."""
    import torch
    import torch.distributed as dist

    from .distributed import reduce_images

    if not dist.is_initialized():
        raise InvalidParameterError(3, "a communicator of size > 1 needs an initialised torch.distributed group")
    t = torch.from_numpy(np.ascontiguousarray(images, dtype=np.float32))
    if dist.get_backend() == "nccl":
        t = t.cuda(device) if device is not None else t.cuda()
    reduce_images(t, dst=0)
    return t.cpu().numpy()


def _synthesize(ctx: Context, opt: NufftSynthesisOptions, dataset, selection, tags, lmn, normalize: bool) -> np.ndarray:
    """One bipp_image_synthesis call over the given selection: images [nImages, nPixel]."""
    n_beam = dataset.num_beam()
    n_samples = len(selection[tags[0]])
    ids = np.zeros((len(tags), max(n_samples, 1)), dtype=np.uint64)
    keep = []
    ptrs = (C.c_void_p * (len(tags) * max(n_samples, 1)))()
    for ti, tag in enumerate(tags):
        sel = selection[tag]
        if len(sel) == 0:
            raise InvalidParameterError(3, "Empty selection")
        if len(sel) != n_samples:
            raise InvalidParameterError(3, "Selection must contain the same sample ids for all images.")
        for k, (sid, ev) in enumerate(sel.items()):
            ev = np.ascontiguousarray(ev, dtype=np.float32)
            if ev.shape[0] != n_beam:
                raise InvalidParameterError(3, "Number of eigenvalues in selection does not match number of beams.")
            keep.append(ev)
            ids[ti, k] = int(sid)
            ptrs[ti * n_samples + k] = ev.ctypes.data
    lmn = np.asfortranarray(lmn, dtype=np.float32)
    n_pixel = lmn.shape[0]
    images = np.zeros((len(tags), n_pixel), dtype=np.float32)

    # dataset callbacks (kept alive for the duration of the call)
    def f_ns(_):
        return dataset.num_samples()

    def f_na(_):
        return dataset.num_antenna()

    def f_nb(_):
        return dataset.num_beam()

    def f_vec(_, i, vptr, ldv):
        v = np.asarray(dataset.eig_vec(i), dtype=np.complex64)
        dst = np.ctypeslib.as_array(C.cast(vptr, C.POINTER(C.c_float)), shape=(2 * ldv * v.shape[1],))
        dst = dst.view(np.complex64).reshape((v.shape[1], ldv)).T
        dst[: v.shape[0], :] = v

    def f_val(_, i, dptr):
        d = np.asarray(dataset.eig_val(i), dtype=np.float32)
        np.ctypeslib.as_array(dptr, shape=(d.shape[0],))[:] = d

    def f_uvw(_, i, uptr, ld):
        u = np.asarray(dataset.uvw(i), dtype=np.float32)
        dst = np.ctypeslib.as_array(uptr, shape=(3 * ld,)).reshape((3, ld)).T
        dst[: u.shape[0], :] = u

    def f_wl(_, i):
        return float(dataset.wl(i))

    def f_sc(_, i):
        return float(dataset.scale(i))

    cbs = _lib.DatasetCallbacks(None, _lib.NUM_SAMPLES_FN(f_ns), _lib.NUM_SAMPLES_FN(f_na),
                                _lib.NUM_SAMPLES_FN(f_nb), _lib.EIG_VEC_FN(f_vec), _lib.EIG_VAL_FN(f_val),
                                _lib.UVW_FN(f_uvw), _lib.SCALAR_FN(f_wl), _lib.SCALAR_FN(f_sc))
    o = opt._c()
    o.normalizeImage = 1 if normalize else 0
    check(ctx._lib.bipp_image_synthesis(ctx.handle, C.byref(o), C.byref(cbs), len(tags), n_samples, _ptr(ids),
                                        C.cast(ptrs, C.c_void_p), n_pixel, _ptr(lmn), n_pixel, _ptr(images)))
    return images


# --- batched pipeline ---------------------------------------------------------------------

_FILTERS = {"lsq": 0, "std": 1, "sqrt": 2, "inv": 3, "inv_sqrt": 4}
# arithmetic of the virtual-visibility products (bipp_pipeline_config.vvPrecision)
VV_PRECISION = {"tf32x3": 0, "bf16x3": 1, "fp32": 2, "fp64": 3}


class Pipeline:
    """Batched Bluebild pipeline: S, antenna positions, wavelength per time step ->
    eigensolve -> energy levels -> virtual visibilities -> NUFFT images.

    lattice: (gridA, gridB, l0, m0, A_l, B_l, A_m, B_m) with pixel (a, b) at
    l = l0 + a A_l + b B_l, m = m0 + a A_m + b B_m; pixel_n: [gridA * gridB] FP64;
    uvw_basis: 3x3 (columns U, V, W in the frame of the positions);
    intervals: [nLevels, 2]; mode "batched" (one NUFFT per call) or "plain" (one NUFFT
    per step and level); vv_precision: arithmetic of VV = X diag(s) X^H, "tf32x3" or
    "bf16x3" (tensor cores, split operands, FP32 accumulation), "fp32" (CUDA cores) or
    "fp64"."""

    def __init__(self, ctx: Context, n_antenna: int, intervals, lattice, pixel_n, uvw_basis, tolerance=1e-5,
                 filter="lsq", chunk_steps=256, max_steps=0, mode="batched", vv_precision="tf32x3"):
        self.ctx = ctx
        self.n_antenna = int(n_antenna)
        self.intervals = np.ascontiguousarray(intervals, dtype=np.float64).reshape(-1, 2)
        self.n_levels = self.intervals.shape[0]
        self.grid = (int(lattice[0]), int(lattice[1]))
        self.pixel_n = np.ascontiguousarray(pixel_n, dtype=np.float64)
        self.basis = np.asfortranarray(uvw_basis, dtype=np.float64)
        cfg = _lib.PipelineConfig()
        cfg.nAntenna = self.n_antenna
        cfg.nLevels = self.n_levels
        cfg.intervals = self.intervals.ctypes.data_as(C.POINTER(C.c_double))
        cfg.filter = _FILTERS[filter]
        cfg.tolerance = float(tolerance)
        cfg.gridA, cfg.gridB = self.grid
        for i in range(6):
            cfg.lattice[i] = float(lattice[2 + i])
        cfg.pixelN = self.pixel_n.ctypes.data_as(C.POINTER(C.c_double))
        cfg.uvwBasis = self.basis.ctypes.data_as(C.POINTER(C.c_double))
        cfg.chunkSteps = int(chunk_steps)
        cfg.maxSteps = int(max_steps)
        cfg.mode = 0 if mode == "batched" else 1
        cfg.vvPrecision = VV_PRECISION[vv_precision]
        h = C.c_void_p()
        check(ctx._lib.bipp_pipeline_create(ctx.handle, C.byref(cfg), C.byref(h)))
        self.handle = h

    def process(self, s, xyz, wl):
        """s [T, N, N] complex64 visibility matrices (s[t][i, j]), xyz [T, N, 3] float64
        positions, wl [T] float64 (host arrays). The matrices are handed to the library in
        its column-major layout."""
        s = np.ascontiguousarray(np.transpose(np.asarray(s, dtype=np.complex64), (0, 2, 1)))
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        wl = np.ascontiguousarray(wl, dtype=np.float64)
        check(self.ctx._lib.bipp_pipeline_process(self.handle, s.shape[0], _ptr(s), _ptr(xyz), _ptr(wl), 0))

    def process_device(self, n_steps, s_ptr, xyz_ptr, wl_ptr):
        """process() on device pointers (e.g. torch data_ptr()); s_ptr holds each step's
        matrix in column-major order ([T][N][N] with element (i, j) at i + j N)."""
        check(self.ctx._lib.bipp_pipeline_process(self.handle, int(n_steps), C.c_void_p(s_ptr), C.c_void_p(xyz_ptr),
                                                  C.c_void_p(wl_ptr), 1))

    def process_host_ptr(self, n_steps, s_ptr, xyz_ptr, wl_ptr):
        """process() on host pointers already in the library layout (s column-major per
        step); the call copies them to the device (pinned memory gives full bandwidth)."""
        check(self.ctx._lib.bipp_pipeline_process(self.handle, int(n_steps), C.c_void_p(s_ptr), C.c_void_p(xyz_ptr),
                                                  C.c_void_p(wl_ptr), 0))

    def stage_host_ptr(self, n_steps, s_ptr, xyz_ptr, wl_ptr):
        """Copy a batch of host inputs (library layout, pinned for an asynchronous copy) into
        a staging slot and return at once (bipp_pipeline_stage)."""
        check(self.ctx._lib.bipp_pipeline_stage(self.handle, int(n_steps), C.c_void_p(s_ptr), C.c_void_p(xyz_ptr),
                                                C.c_void_p(wl_ptr)))

    def process_staged(self):
        """Process the oldest staged batch (bipp_pipeline_process_staged)."""
        check(self.ctx._lib.bipp_pipeline_process_staged(self.handle))

    def images_ptr(self, ptr, normalize=True, on_device=False):
        check(self.ctx._lib.bipp_pipeline_images(self.handle, C.c_void_p(ptr), 1 if normalize else 0,
                                                 1 if on_device else 0))

    def images(self, normalize=True):
        out = np.zeros((self.n_levels, self.grid[0] * self.grid[1]), dtype=np.float32)
        check(self.ctx._lib.bipp_pipeline_images(self.handle, _ptr(out), 1 if normalize else 0, 0))
        return out

    def images_device(self, ptr, normalize=True):
        check(self.ctx._lib.bipp_pipeline_images(self.handle, C.c_void_p(ptr), 1 if normalize else 0, 1))

    def reset(self):
        check(self.ctx._lib.bipp_pipeline_reset(self.handle))

    def last_eigenvalues(self, n_steps):
        d = np.zeros((n_steps, self.n_antenna), dtype=np.float64)
        nr = np.zeros(n_steps, dtype=np.int32)
        check(self.ctx._lib.bipp_pipeline_last_eigenvalues(self.handle, _ptr(d), _ptr(nr)))
        return d, nr

    def stage_times(self, enable: Optional[bool] = None):
        ms = np.zeros(7, dtype=np.float64)
        check(self.ctx._lib.bipp_pipeline_stage_times(self.handle, -1 if enable is None else int(enable), _ptr(ms)))
        return ms

    def kernel_times(self):
        """Eigensolver kernel times (ms): prep, cholesky, trinv, reduction GEMMs, hetrd,
        tridiagonal eigenpairs, back-transform, Linv^H Y GEMM."""
        ms = np.zeros(8, dtype=np.float64)
        check(self.ctx._lib.bipp_pipeline_kernel_times(self.handle, _ptr(ms)))
        return ms

    def nufft_stats(self):
        """Last NUFFT: dict(points, slabs, grid_bytes, items, nx, ny, nw, W, split_tiles)."""
        st = np.zeros(9, dtype=np.int64)
        check(self.ctx._lib.bipp_pipeline_nufft_stats(self.handle, _ptr(st)))
        return dict(zip(["points", "slabs", "grid_bytes", "items", "nx", "ny", "nw", "W", "split_tiles"],
                        [int(x) for x in st]))

    def autotune(self, n_steps, s_ptr, xyz_ptr, wl_ptr, on_device=True, repeats=1):
        """Time the candidate launch parameters on these steps (pointers as
        process_device / process_host_ptr), keep the fastest in the process-wide tuning
        table, and return the per-candidate times (device ms of the stage each parameter
        changes) with the choices. The images are left as they were."""
        import json

        buf = C.create_string_buffer(8192)
        check(self.ctx._lib.bipp_autotune_pipeline(self.handle, int(n_steps), C.c_void_p(s_ptr), C.c_void_p(xyz_ptr),
                                                   C.c_void_p(wl_ptr), 1 if on_device else 0, int(repeats), buf,
                                                   len(buf)))
        return json.loads(buf.value.decode())

    def close(self):
        if getattr(self, "handle", None):
            self.ctx._lib.bipp_pipeline_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --- tuning table of launch parameters ------------------------------------------------------

def tuning_get(name: str) -> int:
    v = C.c_int()
    check(_lib.load().bipp_tuning_get(name.encode(), C.byref(v)))
    return v.value


def tuning_set(name: str, value: int) -> None:
    check(_lib.load().bipp_tuning_set(name.encode(), int(value)))


def tuning_describe() -> dict:
    """{name: {"value", "candidates", "meaning"}} of every tunable launch parameter."""
    buf = C.create_string_buffer(8192)
    check(_lib.load().bipp_tuning_describe(buf, len(buf)))
    out = {}
    for line in buf.value.decode().splitlines():
        name, value, rest = line.split(" ", 2)
        cands, meaning = rest[1:].split("] ", 1)
        out[name] = {"value": int(value), "candidates": [int(c) for c in cands.split()], "meaning": meaning}
    return out


def tuning_save(path: str) -> None:
    check(_lib.load().bipp_tuning_save(str(path).encode()))


def tuning_load(path: str) -> None:
    check(_lib.load().bipp_tuning_load(str(path).encode()))


def tuning_reset() -> None:
    check(_lib.load().bipp_tuning_reset())
