"""Device-resident pipeline: the Subtractor's stage sequence with every image
kept in HBM between stages (C ABI calls in DGPU_MEM_DEVICE mode).

PyTorch provides the device buffers and the stream (plumbing only); every
stage is a libdelta_gpu kernel sequence. Only the small per-stage results
(stamp lists, theta, PSF taps, catalog rows) come back to the host, as in the
reference's own data flow.
"""

from __future__ import annotations

import ctypes
import os
import threading
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np

from . import _core, _lib
from ._lib import check, context
from ._log import logger

try:  # plumbing only
    import torch
except ImportError:  # pragma: no cover - the image ships torch
    torch = None

MEM_DEVICE = _lib.MEM_DEVICE


def available() -> bool:
    return torch is not None and torch.cuda.is_available()


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


@dataclass
class DeviceFrame:
    """Science / reference layers resident on the device (float32 / uint8, H x W)."""

    science: object
    reference: object
    science_var: object = None
    reference_var: object = None
    science_mask: object = None
    reference_mask: object = None

    # Upload of the variance layers still in flight (serialized uploads only):
    # wait_variances() orders the current stream after it.
    variances_ready: object = None

    @property
    def shape(self):
        return tuple(self.science.shape)

    def wait_variances(self) -> None:
        if self.variances_ready is not None:
            torch.cuda.current_stream().wait_event(self.variances_ready)

    def finish_upload(self) -> None:
        """Block until every layer has arrived (the host arrays may then go)."""
        if self.variances_ready is not None:
            self.variances_ready.synchronize()

    @classmethod
    def from_numpy(cls, sci, ref, svar=None, rvar=None, smask=None, rmask=None, device=None, non_blocking=False,
                   serialize=False):
        """Upload the layers. With serialize, the copies of frames uploading from
        several host threads go in call order through one upload stream of the
        device, so each frame's layers arrive at the full host-link rate instead
        of every frame's upload sharing the link with the others. The current
        stream then waits for the science, reference and mask layers (stamp
        selection needs no more), and wait_variances() for the rest; the host
        arrays must stay unchanged until finish_upload() or the frame's work has
        run."""
        dev = device or torch.device("cuda", torch.cuda.current_device())

        def up(a, dt):
            if a is None:
                return None
            t = torch.from_numpy(np.ascontiguousarray(a, dtype=dt))
            return t.to(dev, non_blocking=non_blocking)

        if not serialize:
            return cls(up(sci, np.float32), up(ref, np.float32), up(svar, np.float32), up(rvar, np.float32),
                       up(smask, np.uint8), up(rmask, np.uint8))
        # Pageable layers are first copied into pinned buffers by several host
        # threads (outside the lock, so while another frame's layers cross the
        # link): the driver's own pageable path stages them through one thread.
        host = [_pinned_layer(a, dt) for a, dt in ((sci, np.float32), (ref, np.float32), (smask, np.uint8),
                                                   (rmask, np.uint8), (svar, np.float32), (rvar, np.float32))]

        def send(t):
            return None if t is None else t.to(dev, non_blocking=True)

        cur = torch.cuda.current_stream(dev)
        up_s = _upload_stream(dev)
        with _UPLOAD_LOCK:  # one frame's copies stay together on the shared stream
            up_s.wait_stream(cur)
            with torch.cuda.stream(up_s):
                s_, r_, sm_, rm_ = (send(t) for t in host[:4])
                first = torch.cuda.Event()
                first.record(up_s)
                sv_, rv_ = (send(t) for t in host[4:])
                rest = torch.cuda.Event()
                rest.record(up_s)
        cur.wait_event(first)
        for t in (s_, r_, sv_, rv_, sm_, rm_):
            if t is not None:  # the frame's work runs on cur: no reuse of the memory before it has
                t.record_stream(cur)
        return cls(s_, r_, sv_, rv_, sm_, rm_, variances_ready=rest)


_CUDA_STREAM_LEGACY = 0x1  # cudaStreamLegacy: handle 0 would select the context's own stream
_UPLOAD_LOCK = threading.Lock()
_XFER_STREAMS: dict = {}
_STAGE_CHUNK = 8 << 20
_STAGE_MIN = 1 << 20
_stage_pool: list = []
_stage_lock = threading.Lock()


def _stage_threads() -> ThreadPoolExecutor:
    with _stage_lock:
        if not _stage_pool:
            n = max(2, min(8, (os.cpu_count() or 2) // 2))
            _stage_pool.append(ThreadPoolExecutor(max_workers=n, thread_name_prefix="delta-b200-stage"))
        return _stage_pool[0]


def _pinned_layer(a, dt):
    """A CPU tensor of layer `a` (as dtype dt) in pinned memory: `a` itself when
    it already is (or is small), else a pinned copy made in 8 MB pieces by the
    staging threads. The pinned copy comes from torch's caching host
    allocator, which reuses it only after the transfers queued from it have
    run."""
    if a is None:
        return None
    h = np.ascontiguousarray(a, dtype=dt)
    t = torch.from_numpy(h)
    if h.nbytes < _STAGE_MIN or t.is_pinned():
        return t
    buf = torch.empty(h.shape, dtype=t.dtype, pin_memory=True)
    dst, src = buf.numpy().reshape(-1), h.reshape(-1)
    step = max(1, _STAGE_CHUNK // h.itemsize)
    futs = [_stage_threads().submit(np.copyto, dst[o:o + step], src[o:o + step]) for o in range(0, src.size, step)]
    for f in futs:
        f.result()
    return buf


def _upload_stream(dev):
    """The device's one stream for serialized frame uploads."""
    with _UPLOAD_LOCK:
        s = _XFER_STREAMS.get(dev.index)
        if s is None:
            s = _XFER_STREAMS[dev.index] = torch.cuda.Stream(device=dev)
        return s


def _ctx_on_torch_stream():
    """The thread's context, ordered on torch's current stream (the layers are
    torch tensors written there)."""
    ctx = context()
    ctx.set_stream(torch.cuda.current_stream().cuda_stream or _CUDA_STREAM_LEGACY)
    return ctx


def select_stamps(frame: DeviceFrame, sub, catalog=None) -> dict:
    ctx = _ctx_on_torch_stream()
    h, w = frame.shape
    cx = cy = None
    ncat = 0
    if catalog is not None:
        cat = np.asarray(catalog, dtype=np.int32)
        cx = np.ascontiguousarray(cat[:, 0])
        cy = np.ascontiguousarray(cat[:, 1])
        ncat = cx.size
    p = _core._detect_params(sub.stamp_radius, sub.threshold_sigma, sub.max_stamps, sub.saturation, 0, 0,
                             sub.fwhm_radius, sub.match_radius)
    cap = max(int(sub.max_stamps), ncat, 1)
    x = np.zeros(cap, np.int32)
    y = np.zeros(cap, np.int32)
    fs = np.zeros(cap)
    fr = np.zeros(cap)
    ms, mr = ctypes.c_double(), ctypes.c_double()
    dref, n = ctypes.c_int(), ctypes.c_int()
    check(_lib.lib().dgpu_select_stamps(
        ctx.handle, MEM_DEVICE, ctypes.c_int64(w), ctypes.c_int64(h), _p(frame.science), _p(frame.reference),
        _p(frame.science_mask), _p(frame.reference_mask), _lib.ptr(cx), _lib.ptr(cy), int(ncat), ctypes.byref(p),
        cap, _lib.ptr(x), _lib.ptr(y), _lib.ptr(fs), _lib.ptr(fr), ctypes.byref(ms), ctypes.byref(mr),
        ctypes.byref(dref), ctypes.byref(n)), ctx.handle)
    k = n.value
    return {"x": x[:k].copy(), "y": y[:k].copy(), "fwhm_science": fs[:k].copy(), "fwhm_reference": fr[:k].copy(),
            "median_fwhm_science": ms.value, "median_fwhm_reference": mr.value,
            "direction": "reference" if dref.value else "science"}


def fit_kernel(target, conv, tvar, cvar, tmask, cmask, knots, stamp_x, stamp_y, sub, beta) -> dict:
    ctx = _ctx_on_torch_stream()
    h, w = target.shape
    k = np.ascontiguousarray(knots, np.float64)
    sx = np.ascontiguousarray(stamp_x, np.int32)
    sy = np.ascontiguousarray(stamp_y, np.int32)
    grid = np.ascontiguousarray(sub.lambda_grid, np.float64)
    nc = (sub.n_max + 1) * (sub.n_max + 2) // 2
    res, bufs = _core._gls_struct((nc + 1) * k.shape[0], grid.size, nc, sx.size)
    check(_lib.lib().dgpu_fit_kernel(
        ctx.handle, MEM_DEVICE, ctypes.c_int64(w), ctypes.c_int64(h), _p(target), _p(conv), _p(tvar), _p(cvar),
        _p(tmask), _p(cmask), _lib.ptr(k), k.shape[0], _lib.ptr(sx), _lib.ptr(sy), int(sx.size),
        int(sub.stamp_radius), ctypes.c_double(beta), int(sub.n_max), int(sub.radius), _lib.ptr(grid),
        int(grid.size), ctypes.c_double(sub.clip_sigma), int(sub.clip_iterations), int(sub.min_stamps),
        int(sub.cv_folds), _core.PRECISIONS[sub.precision], ctypes.byref(res)), ctx.handle)
    out = _core._gls_dict(res, bufs)
    nt = int(res.n_stamps_total)
    out.update({
        "component_sums": bufs["component_sums"][:nc].copy(), "n_pixels": int(res.n_pixels),
        "n_stamps_used": int(res.n_stamps_used), "n_stamps_total": nt,
        "n_stamps_rejected": int(res.n_stamps_rejected), "reduced_chi2": float(res.reduced_chi2),
        "cv_exact_design_bytes": int(res.cv_exact_design_bytes), "stamp_x": bufs["stamp_x"][:nt].copy(),
        "stamp_y": bufs["stamp_y"][:nt].copy(), "stamp_chi2": bufs["stamp_chi2"][:nt].copy(),
        "stamp_accepted": bufs["stamp_accepted"][:nt].copy()})
    return out


def subtract(target, conv, tvar, cvar, tmask, cmask, solution, saturation):
    ctx = _ctx_on_torch_stream()
    h, w = target.shape
    model, keep = _core._model(solution.knots, solution.theta, solution.beta, solution.n_max, solution.radius)
    diff = torch.empty((h, w), dtype=torch.float32, device=target.device)
    want_var = tvar is not None or cvar is not None
    want_mask = tmask is not None or cmask is not None or saturation > 0
    var = torch.empty_like(diff) if want_var else None
    mask = torch.empty((h, w), dtype=torch.uint8, device=target.device) if want_mask else None
    hv, hm = ctypes.c_int(), ctypes.c_int()
    check(_lib.lib().dgpu_subtract(ctx.handle, MEM_DEVICE, ctypes.c_int64(w), ctypes.c_int64(h), _p(target),
                                   _p(conv), _p(tvar), _p(cvar), _p(tmask), _p(cmask), ctypes.byref(model),
                                   ctypes.c_double(saturation), _p(diff), _p(var), _p(mask), ctypes.byref(hv),
                                   ctypes.byref(hm)), ctx.handle)
    return diff, var if hv.value else None, mask if hm.value else None


def variance_rescale_factor(diff, var, mask) -> float:
    """_variance_rescale_factor (median(D^2 / Var) / median(chi2_1) over the good
    pixels) with the median selected on the device: no frame leaves HBM."""
    from .pipeline import _MEDIAN_CHI2_1

    ctx = _ctx_on_torch_stream()
    med, cnt = ctypes.c_double(), ctypes.c_int64()
    check(_lib.lib().dgpu_z2_median(ctx.handle, MEM_DEVICE, ctypes.c_int64(diff.numel()), _p(diff), _p(var),
                                    _p(mask), ctypes.byref(med), ctypes.byref(cnt)), ctx.handle)
    return 1.0 if cnt.value == 0 else float(med.value / _MEDIAN_CHI2_1)


def scale_(t, factor: float) -> None:
    """t *= factor in place on the device (library kernel, float32 product)."""
    ctx = _ctx_on_torch_stream()
    check(_lib.lib().dgpu_scale(ctx.handle, MEM_DEVICE, _p(t), ctypes.c_int64(t.numel()), ctypes.c_double(factor)),
          ctx.handle)


def fill_(t, value: float) -> None:
    """t[:] = value on the device (library kernel)."""
    ctx = _ctx_on_torch_stream()
    check(_lib.lib().dgpu_fill(ctx.handle, MEM_DEVICE, _p(t), ctypes.c_int64(t.numel()), ctypes.c_double(value)),
          ctx.handle)


def negate(t) -> None:
    ctx = _ctx_on_torch_stream()
    check(_lib.lib().dgpu_negate(ctx.handle, MEM_DEVICE, _p(t), ctypes.c_int64(t.numel())), ctx.handle)


class EarlyDownload:
    """Device-to-host copies of some final products, started on the calling
    thread's download stream while the frame's remaining stages compute."""

    def __init__(self, products: dict):
        cur = torch.cuda.current_stream()
        s = _thread_download_stream()
        s.wait_stream(cur)
        self.host = {}
        with torch.cuda.stream(s):
            for key, t in products.items():
                if t is None:
                    self.host[key] = None
                    continue
                t = t.contiguous()
                h = torch.empty(tuple(t.shape), dtype=t.dtype, pin_memory=True)
                h.copy_(t, non_blocking=True)
                t.record_stream(s)
                self.host[key] = h
        self.done = torch.cuda.Event()
        self.done.record(s)


def download(out: dict, early: EarlyDownload | None = None) -> dict:
    """Copy the image products of run()/apply() into pinned host memory;
    returns {name: ndarray | None}. The copies go through the copy engine
    (dgpu_copy_to_host, or `early`'s copies for the products it holds); the
    library's own small read-backs reach the host by SM stores, so frames
    computing on other streams do not wait behind a 200 MB download."""
    ctx = _ctx_on_torch_stream()
    pinned = {}
    for key in ("difference", "variance", "mask", "score"):
        if early is not None and key in early.host:
            pinned[key] = early.host[key]
            continue
        t = out.get(key)
        if t is None:
            pinned[key] = None
            continue
        t = t.contiguous()
        hbuf = torch.empty(tuple(t.shape), dtype=t.dtype, pin_memory=True)
        check(_lib.lib().dgpu_copy_to_host(ctx.handle, ctypes.c_void_p(hbuf.data_ptr()), _p(t),
                                           ctypes.c_int64(t.numel() * t.element_size())), ctx.handle)
        pinned[key] = hbuf
    torch.cuda.current_stream().synchronize()
    if early is not None:
        early.done.synchronize()
    return {k: (None if v is None else v.numpy()) for k, v in pinned.items()}


def download_bytes(out: dict) -> int:
    return sum(out[k].numel() * out[k].element_size() for k in ("difference", "variance", "mask", "score")
               if out.get(k) is not None)


def decorrelate(diff, solution, tvar, cvar, block):
    ctx = _ctx_on_torch_stream()
    h, w = diff.shape
    model, keep = _core._model(solution.knots, solution.theta, solution.beta, solution.n_max, solution.radius)
    out_d = torch.empty_like(diff)
    out_v = torch.empty_like(diff)
    check(_lib.lib().dgpu_decorrelate(ctx.handle, MEM_DEVICE, ctypes.c_int64(w), ctypes.c_int64(h), _p(diff),
                                      ctypes.byref(model), _p(tvar), _p(cvar), int(block), 0, _p(out_d), _p(out_v)),
          ctx.handle)
    return out_d, out_v


def estimate_psf(image, xs, ys, radius) -> np.ndarray:
    ctx = _ctx_on_torch_stream()
    h, w = image.shape
    x = np.ascontiguousarray(xs, np.int32)
    y = np.ascontiguousarray(ys, np.int32)
    side = 2 * int(radius) + 1
    out = np.empty((side, side), np.float32)
    check(_lib.lib().dgpu_estimate_psf(ctx.handle, MEM_DEVICE, ctypes.c_int64(w), ctypes.c_int64(h), _p(image),
                                       _lib.ptr(x), _lib.ptr(y), int(min(x.size, y.size)), int(radius),
                                       _lib.ptr(out)), ctx.handle)
    return out


def whiten_score_psf(psf, solution, tvar, cvar, block) -> np.ndarray:
    ctx = _ctx_on_torch_stream()
    h, w = tvar.shape
    model, keep = _core._model(solution.knots, solution.theta, solution.beta, solution.n_max, solution.radius)
    p = np.ascontiguousarray(psf, np.float32)
    out = np.empty_like(p)
    check(_lib.lib().dgpu_whiten_score_psf(ctx.handle, MEM_DEVICE, _lib.ptr(p), int(p.shape[0]), ctypes.byref(model),
                                           ctypes.c_int64(w), ctypes.c_int64(h), _p(tvar), _p(cvar), int(block),
                                           _lib.ptr(out)), ctx.handle)
    return out


def matched_filter(image, psf, variance):
    ctx = _ctx_on_torch_stream()
    h, w = image.shape
    p = np.ascontiguousarray(psf, np.float32)
    out = torch.empty_like(image)
    check(_lib.lib().dgpu_matched_filter(ctx.handle, MEM_DEVICE, ctypes.c_int64(w), ctypes.c_int64(h), _p(image),
                                         _lib.ptr(p), int(p.shape[0]), _p(variance), _p(out)), ctx.handle)
    return out


def build_catalog(score, difference, mask, psf, threshold_sigma=5.0, threshold_sigma_dipole=3.0) -> dict:
    from .catalog import _measure_psf_fwhm, _pack

    ctx = _ctx_on_torch_stream()
    h, w = score.shape
    prm = _lib.CatalogParams(float(threshold_sigma), float(threshold_sigma_dipole), _measure_psf_fwhm(psf), 0.3, 3.0,
                             0, 1, 0, 0, 3.0, 0.0, 5000)
    n = ctypes.c_int()
    L = _lib.lib()
    check(L.dgpu_build_catalog(ctx.handle, MEM_DEVICE, ctypes.c_int64(w), ctypes.c_int64(h), _p(score),
                               _p(difference), _p(mask), ctypes.byref(prm), None, None, 0, None, None, 0,
                               ctypes.byref(n)), ctx.handle)
    cols = {name: np.empty(n.value, dt) for name, dt in _lib.CATALOG_COLUMNS}
    cc = _lib.CatalogColumns(*[cols[name].ctypes.data for name, _ in _lib.CATALOG_COLUMNS])
    check(L.dgpu_catalog_fetch(ctx.handle, ctypes.byref(cc), n.value), ctx.handle)
    return _pack(cols)


def run(sub, frame: DeviceFrame, catalog=None, direction=None, early=None) -> dict:
    """One Subtractor.subtract pass on device-resident layers (fit -> subtract ->
    [decorrelate] -> [score + catalog]). Returns device tensors for the images
    and host values for the solution / PSF / catalog."""
    from .pipeline import _default_beta
    from .solution import KernelSolution

    sel = select_stamps(frame, sub, catalog)
    logger.info("selected {} stamps (median FWHM: science={:.2f}, reference={:.2f} px)", len(sel["x"]),
                sel["median_fwhm_science"], sel["median_fwhm_reference"])
    if len(sel["x"]) == 0:
        raise ValueError("no stamps selected; lower threshold_sigma, supply a catalog, or widen match_radius "
                         "if science/reference are astrometrically misregistered")
    if direction is None:
        direction = sel["direction"]
    elif direction not in ("science", "reference"):
        raise ValueError(f"direction must be 'science', 'reference', or None, got {direction!r}")
    if direction == "science":
        target, tvar, tmask = frame.reference, frame.reference_var, frame.reference_mask
        conv, cvar, cmask = frame.science, frame.science_var, frame.science_mask
        sign = -1.0
    else:
        target, tvar, tmask = frame.science, frame.science_var, frame.science_mask
        conv, cvar, cmask = frame.reference, frame.reference_var, frame.reference_mask
        sign = 1.0
    beta = sub.beta if sub.beta is not None else _default_beta(sel["median_fwhm_science"],
                                                                sel["median_fwhm_reference"])
    h, w = frame.shape
    nkx = nky = sub.n_knots
    if sub.spatial_scale is not None and sub.spatial_scale > 0:
        nkx = int(np.clip(round((w - 1) / sub.spatial_scale) + 1, 3, sub.n_knots))
        nky = int(np.clip(round((h - 1) / sub.spatial_scale) + 1, 3, sub.n_knots))
    knots = _core.grid_knots(0.0, 0.0, w - 1.0, h - 1.0, nkx, nky)
    frame.wait_variances()
    fit = fit_kernel(target, conv, tvar, cvar, tmask, cmask, knots, sel["x"], sel["y"], sub, beta)
    logger.info("kernel fit: lambda={:.3g}, eff.dof={:.1f}, reduced chi2={:.3f} ({} stamps used, {} rejected of {}, "
                "{} px)", fit["lambda"], fit["effective_dof"], fit["reduced_chi2"], fit["n_stamps_used"],
                fit["n_stamps_rejected"], fit["n_stamps_total"], fit["n_pixels"])
    solution = KernelSolution(
        beta=beta, n_max=sub.n_max, radius=sub.radius, knots=knots, theta=fit["theta"],
        n_components=fit["n_components"], n_spatial=fit["n_spatial"], lam=fit["lambda"], gcv=fit["gcv"],
        effective_dof=fit["effective_dof"], rss=fit["rss"], component_sums=fit["component_sums"],
        direction=direction, shape=(h, w), reduced_chi2=fit["reduced_chi2"], n_stamps_used=fit["n_stamps_used"],
        n_stamps_rejected=fit["n_stamps_rejected"], stamp_x=fit["stamp_x"], stamp_y=fit["stamp_y"],
        stamp_chi2=fit["stamp_chi2"], stamp_accepted=fit["stamp_accepted"])
    return apply(sub, solution, target, conv, tvar, cvar, tmask, cmask, sign, sel["x"], sel["y"], early)


def apply_solution(sub, solution, frame: DeviceFrame, early=None) -> dict:
    """Subtractor.apply on device-resident layers: a frozen solution, no re-fit."""
    frame.wait_variances()
    if solution.direction == "science":
        return apply(sub, solution, frame.reference, frame.science, frame.reference_var, frame.science_var,
                     frame.reference_mask, frame.science_mask, -1.0, solution.stamp_x, solution.stamp_y, early)
    return apply(sub, solution, frame.science, frame.reference, frame.science_var, frame.reference_var,
                 frame.science_mask, frame.reference_mask, 1.0, solution.stamp_x, solution.stamp_y, early)


def apply(sub, solution, target, conv, tvar, cvar, tmask, cmask, sign, stamp_x, stamp_y, early=None) -> dict:
    """The stages after the fit. `early(products)`, when given, receives the
    difference, variance and mask as soon as they are final (before the score
    and catalog), e.g. to start their download."""
    out_levels = [v for v in (sub.saturation, sub.bright_mask) if v and v > 0]
    out_saturation = min(out_levels) if out_levels else 0.0
    diff, var, mask = subtract(target, conv, tvar, cvar, tmask, cmask, solution, out_saturation)
    if sign < 0:
        negate(diff)
    variance_scale = None
    if sub.rescale_variance and var is not None:
        variance_scale = variance_rescale_factor(diff, var, mask)
        scale_(var, variance_scale)
    whitened, white_var = diff, None
    if sub.decorrelate and tvar is not None and cvar is not None:
        whitened, white_var = decorrelate(diff, solution, tvar, cvar, sub.block)
        if variance_scale is not None:
            scale_(white_var, variance_scale)
    if early is not None:  # these three are final from here on
        early({"difference": whitened, "variance": white_var if white_var is not None else var, "mask": mask})
    score = psf = cat = None
    if sub.score:
        if stamp_x is None or np.asarray(stamp_x).size == 0:
            raise ValueError("score requested but the solution carries no stamp positions for PSF estimation")
        psf = estimate_psf(target, stamp_x, stamp_y, min(sub.stamp_radius, 8))
        if white_var is not None:
            score_var = white_var
            psf = whiten_score_psf(psf, solution, tvar, cvar, sub.block)
        elif var is not None:
            score_var = var
        else:
            score_var = torch.empty_like(whitened)
            fill_(score_var, float(np.var(whitened.cpu().numpy())))
        score = matched_filter(whitened, psf, score_var)
        if sub.source_catalog:
            cat = build_catalog(score, whitened, mask, psf)
    return {"solution": solution, "difference": whitened, "variance": white_var if white_var is not None else var,
            "mask": mask, "score": score, "psf": psf, "catalog": cat, "variance_scale": variance_scale}


# ---------------------------------------------------------------------------
# Several frames in flight: one host thread, one library context and one CUDA
# stream per frame, so the latency-bound phases of one frame (selection, the
# per-lambda solves, single-CTA selects) overlap the bandwidth-bound phases of
# another. Worker threads persist, so their contexts keep their workspace.
# ---------------------------------------------------------------------------

_runners: dict = {}
_runners_lock = threading.Lock()
_tls = threading.local()


def _thread_stream():
    s = getattr(_tls, "stream", None)
    if s is None:
        s = _tls.stream = torch.cuda.Stream()
    return s


def _thread_download_stream():
    s = getattr(_tls, "dl_stream", None)
    if s is None:
        s = _tls.dl_stream = torch.cuda.Stream()
    return s


def runner(n_workers: int) -> ThreadPoolExecutor:
    """The persistent pool of `n_workers` frame workers (one per frame in flight)."""
    n = max(1, int(n_workers))
    with _runners_lock:
        ex = _runners.get(n)
        if ex is None:
            ex = _runners[n] = ThreadPoolExecutor(max_workers=n, thread_name_prefix=f"delta-b200-frame{n}")
        return ex


def on_own_stream(fn, *args, **kwargs):
    """Run fn on the calling worker's stream, after the work already queued on
    the default stream (inputs uploaded there), and wait for it to finish."""
    s = _thread_stream()
    s.wait_stream(torch.cuda.default_stream())
    with torch.cuda.stream(s):
        out = fn(*args, **kwargs)
    s.synchronize()
    return out


def run_batch(sub, frames, catalogs=None, directions=None, max_in_flight: int | None = None) -> list:
    """run() over several device-resident frames with up to `max_in_flight`
    frames processed concurrently; results in input order."""
    frames = list(frames)
    n = len(frames)
    if n == 0:
        return []
    catalogs = list(catalogs) if catalogs is not None else [None] * n
    directions = list(directions) if directions is not None else [None] * n
    ex = runner(max_in_flight or min(n, 4))
    futs = [ex.submit(on_own_stream, run, sub, f, c, d) for f, c, d in zip(frames, catalogs, directions, strict=True)]
    return [f.result() for f in futs]
