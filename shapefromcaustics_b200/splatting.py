"""Torch-facing host layer of the splatting ops: the reference's operator interface over the
C ABI of ``libpds_b200.so``.

``pds_forward`` / ``pds_backward`` keep the signatures, return types (Python lists) and
argument checks of the reference module ``PhotonDifferentialSplatting``
(``PyOptix/PhotonDifferentialSplattig.cpp:12-32``; checks :14-22 and ``PyOptix/utils.hpp:37-41``),
so ``from shapefromcaustics_b200.splatting import pds_forward, pds_backward`` replaces
``from PhotonDifferentialSplatting import pds_forward, pds_backward``
(``model/photon_differential.py:4``). Outputs are allocated here in ``Ep``'s dtype and
device, like the reference's ``th::zeros`` / ``th::empty_like``
(``photon_differentials.cu:118``, ``:225-227``); kernels run on the current CUDA stream.

``SplatPlan`` keeps one photon binning + sort for a forward and its backward. ``BatchedSplat``
runs many simulations of uneven sizes through one plan and one persistent launch per
direction.
"""
import ctypes

import torch

from . import _lib
from ._lib import check, lib

__all__ = ["pds_forward", "pds_backward", "SplatPlan", "BatchedSplat", "default_config",
           "set_default_config"]

_default_cfg = _lib.config()


def default_config():
    return _default_cfg


def set_default_config(**fields):
    """Tuning used by calls that pass no config (``pds_config`` fields; zeros or absent
    fields select the library defaults)."""
    global _default_cfg
    _default_cfg = _lib.config(**fields)


def _check_input(t, name):
    # PyOptix/utils.hpp:37-41
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")


def _check_photons(Ep, xp, Mp, cp, radius, op="pds_forward"):
    for t, n in ((Ep, "Ep"), (xp, "xp"), (Mp, "Mp"), (cp, "cp"), (radius, "radius")):
        _check_input(t, n)
    # PhotonDifferentialSplattig.cpp:19-22
    if Ep.dim() != 1 or xp.dim() != 2 or Mp.dim() != 3 or cp.dim() != 2 or radius.dim() != 1:
        raise RuntimeError(f"Dimensions of tensors for {op} don't match")
    n = Ep.size(0)
    if not (n == xp.size(1) and n == Mp.size(2) and n == cp.size(1) and n == radius.size(0)):
        raise RuntimeError(f"Dimensions of tensors for {op} don't match")
    if cp.size(0) != 1:
        raise RuntimeError("Channel index must be one dimensional!")
    if xp.size(0) != 2:
        raise RuntimeError("Position index must be two dimensional!")
    if Mp.size(0) != 2 or Mp.size(1) != 3:
        raise RuntimeError("Change of basis matrix must be 2x3!")
    if cp.dtype != torch.int64:
        raise RuntimeError(f"expected scalar type Long for cp but found {cp.dtype}")
    for t, nm in ((Ep, "Ep"), (xp, "xp"), (Mp, "Mp"), (radius, "radius")):
        if t.dtype != torch.float32:
            raise RuntimeError(
                f"pds_b200 computes in float32; {nm} has dtype {t.dtype}")
    dev = Ep.device
    for t in (xp, Mp, cp, radius):
        if t.device != dev:
            raise RuntimeError(f"all inputs of {op} must be on the same device")
    return n


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() > 0 else ctypes.c_void_p(0)


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _output_size(output_size):
    s = [int(v) for v in output_size]
    if len(s) != 3:
        raise RuntimeError("output_size must be [C, H, W]")
    return s


def _workspace(n, C, H, W, cfg, device):
    nbytes = lib().pds_workspace_bytes(n, C, H, W, ctypes.byref(cfg))
    return torch.empty(int(nbytes), dtype=torch.uint8, device=device)


class SplatPlan:
    """One binning + sort of a photon set, shared by its forward and backward.

    The plan lives in a device workspace owned by this object; ``forward`` and ``backward``
    must be called with the same photon tensors (unchanged) that built it.
    """

    def __init__(self, Ep, xp, Mp, cp, radius, output_size, max_pixel_radius, config=None):
        n = _check_photons(Ep, xp, Mp, cp, radius)
        self.n = n
        self.C, self.H, self.W = _output_size(output_size)
        self.mpr = int(max_pixel_radius)
        self.cfg = config if config is not None else _default_cfg
        self.device = Ep.device
        self.inputs = (Ep, xp, Mp, cp, radius)
        with torch.cuda.device(self.device):
            self.ws = _workspace(n, self.C, self.H, self.W, self.cfg, self.device)
            check(lib().pds_plan_f32(*(_ptr(t) for t in self.inputs), n, self.C, self.H,
                                     self.W, self.mpr, _ptr(self.ws), self.ws.numel(),
                                     ctypes.byref(self.cfg), _stream(self.device)))

    def forward(self, out=None):
        if out is None:
            out = torch.empty((self.C, self.H, self.W), dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            check(lib().pds_forward_planned_f32(*(_ptr(t) for t in self.inputs), self.n, self.C,
                                                self.H, self.W, self.mpr, _ptr(out),
                                                _ptr(self.ws), self.ws.numel(),
                                                ctypes.byref(self.cfg), _stream(self.device)))
        return out

    def backward(self, grad_pds, out=None, records=False):
        """[grad_Ep, grad_xp, grad_Mp]; with ``records`` the gradients stay in the plan's
        workspace as per-photon records (for ``plate.refract_backward_planned``) and None is
        returned."""
        _check_input(grad_pds, "grad_pds")
        if tuple(grad_pds.shape) != (self.C, self.H, self.W) or grad_pds.dtype != torch.float32:
            raise RuntimeError("grad_pds must be a float32 tensor of the forward's output_size")
        Ep, xp, Mp = self.inputs[:3]
        if records:
            gE = gx = gM = None
        else:
            if out is None:
                out = (torch.empty_like(Ep), torch.empty_like(xp), torch.empty_like(Mp))
            gE, gx, gM = out
        with torch.cuda.device(self.device):
            check(lib().pds_backward_planned_f32(_ptr(grad_pds), *(_ptr(t) for t in self.inputs),
                                                 self.n, self.C, self.H, self.W, self.mpr,
                                                 _ptr(gE), _ptr(gx), _ptr(gM), _ptr(self.ws),
                                                 self.ws.numel(), ctypes.byref(self.cfg),
                                                 _stream(self.device)))
        return None if records else [gE, gx, gM]


def pds_forward(Ep, xp, Mp, cp, radius, output_size, max_pixel_radius):
    """``PhotonDifferentialSplatting.pds_forward`` (PhotonDifferentialSplattig.cpp:12-25):
    splats the photons into a new ``[C,H,W]`` image and returns ``[image]``."""
    n = _check_photons(Ep, xp, Mp, cp, radius)
    C, H, W = _output_size(output_size)
    cfg = _default_cfg
    with torch.cuda.device(Ep.device):
        out = torch.empty((C, H, W), dtype=Ep.dtype, device=Ep.device)
        ws = _workspace(n, C, H, W, cfg, Ep.device)
        check(lib().pds_forward_f32(_ptr(Ep), _ptr(xp), _ptr(Mp), _ptr(cp), _ptr(radius), n, C,
                                    H, W, int(max_pixel_radius), _ptr(out), _ptr(ws), ws.numel(),
                                    ctypes.byref(cfg), _stream(Ep.device)))
    return [out]


def pds_backward(grad_pds, Ep, xp, Mp, cp, radius, max_pixel_radius):
    """``PhotonDifferentialSplatting.pds_backward`` (PhotonDifferentialSplattig.cpp:27-32):
    returns ``[grad_Ep, grad_xp, grad_Mp]`` (``grad_Mp[:, 2] == 0``)."""
    _check_input(grad_pds, "grad_pds")
    n = _check_photons(Ep, xp, Mp, cp, radius, op="pds_backward")
    if grad_pds.dim() != 3 or grad_pds.dtype != torch.float32 or grad_pds.device != Ep.device:
        raise RuntimeError("grad_pds must be a float32 [C,H,W] tensor on the inputs' device")
    C, H, W = (int(v) for v in grad_pds.shape)
    cfg = _default_cfg
    with torch.cuda.device(Ep.device):
        gE, gx, gM = torch.empty_like(Ep), torch.empty_like(xp), torch.empty_like(Mp)
        ws = _workspace(n, C, H, W, cfg, Ep.device)
        check(lib().pds_backward_f32(_ptr(grad_pds), _ptr(Ep), _ptr(xp), _ptr(Mp), _ptr(cp),
                                     _ptr(radius), n, C, H, W, int(max_pixel_radius), _ptr(gE),
                                     _ptr(gx), _ptr(gM), _ptr(ws), ws.numel(),
                                     ctypes.byref(cfg), _stream(Ep.device)))
    return [gE, gx, gM]


class BatchedSplat:
    """Many simulations of uneven photon counts and image sizes in one launch sequence.

    ``sims`` is a list of ``(n_photons, (C, H, W))``. Photon tensors passed to ``plan`` are
    the simulations' photons concatenated in order (``Ep[Ntot]``, ``xp[2,Ntot]``,
    ``Mp[2,3,Ntot]``, ``cp[1,Ntot]``, ``radius[Ntot]``). Images live in one flat buffer;
    ``images(flat)`` returns per-simulation views. The reference runs the simulations one
    after another (``shape_from_caustics.py:351-353``).
    """

    def __init__(self, sims, max_pixel_radius, device, config=None):
        self.cfg = config if config is not None else _default_cfg
        self.mpr = int(max_pixel_radius)
        self.device = torch.device(device)
        if self.device.type == "cuda" and self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        n_sims = len(sims)
        table = (_lib.PdsSim * n_sims)()
        begin, off = 0, 0
        self.shapes, self.offsets, self.counts = [], [], []
        for s, (n, shape) in enumerate(sims):
            C, H, W = (int(v) for v in shape)
            table[s].photon_begin = begin
            table[s].n_photons = int(n)
            table[s].image_offset = off
            table[s].channels, table[s].height, table[s].width = C, H, W
            self.shapes.append((C, H, W))
            self.offsets.append(off)
            self.counts.append(int(n))
            begin += int(n)
            off += C * H * W
        self.n_total = begin
        self.image_elems = off
        nt = ctypes.c_int64(0)
        check(lib().pds_batch_layout(table, n_sims, ctypes.byref(self.cfg), ctypes.byref(nt)))
        self.n_tiles = nt.value
        self.n_sims = n_sims
        raw = bytes(table)
        self.table_dev = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(self.device)
        nbytes = lib().pds_batch_workspace_bytes(self.n_total, self.n_tiles, ctypes.byref(self.cfg))
        self.ws = torch.empty(int(nbytes), dtype=torch.uint8, device=self.device)
        self.inputs = None

    def _common(self):
        return (self.n_total, _ptr(self.table_dev), self.n_sims, self.n_tiles)

    def plan(self, Ep, xp, Mp, cp, radius):
        n = _check_photons(Ep, xp, Mp, cp, radius)
        if n != self.n_total:
            raise RuntimeError(f"batch expects {self.n_total} photons, got {n}")
        self.inputs = (Ep, xp, Mp, cp, radius)
        with torch.cuda.device(self.device):
            check(lib().pds_batch_plan_f32(*(_ptr(t) for t in self.inputs), *self._common(),
                                           self.mpr, _ptr(self.ws), self.ws.numel(),
                                           ctypes.byref(self.cfg), _stream(self.device)))

    def _planned(self, op):
        if self.inputs is None:
            raise RuntimeError(f"BatchedSplat.{op}() called before plan()")

    def _check_flat(self, t, name):
        if not (t.is_cuda and t.device == self.device):
            raise RuntimeError(f"{name} must be a CUDA tensor on {self.device}")
        if t.dtype != torch.float32:
            raise RuntimeError(f"{name} must be float32, got {t.dtype}")
        if t.numel() != self.image_elems or not t.is_contiguous():
            raise RuntimeError(f"{name} must be a contiguous flat buffer of the batch's "
                               f"{self.image_elems} image elements")

    def forward(self, out=None):
        self._planned("forward")
        if out is None:
            out = torch.empty(self.image_elems, dtype=torch.float32, device=self.device)
        self._check_flat(out, "out")
        with torch.cuda.device(self.device):
            check(lib().pds_batch_forward_planned_f32(*(_ptr(t) for t in self.inputs),
                                                      *self._common(), self.image_elems,
                                                      self.mpr, _ptr(out), _ptr(self.ws),
                                                      self.ws.numel(), ctypes.byref(self.cfg),
                                                      _stream(self.device)))
        return out

    def backward(self, grad_flat, out=None, records=False):
        """(grad_Ep, grad_xp, grad_Mp) of the batch's photons; with ``records`` the gradients
        stay in the plan's workspace as per-photon records (for
        ``plate.BatchedPlate.backward``) and None is returned."""
        self._planned("backward")
        self._check_flat(grad_flat, "grad")
        Ep, xp, Mp = self.inputs[:3]
        if records:
            gE = gx = gM = None
        else:
            if out is None:
                out = (torch.empty_like(Ep), torch.empty_like(xp), torch.empty_like(Mp))
            gE, gx, gM = out
        with torch.cuda.device(self.device):
            check(lib().pds_batch_backward_planned_f32(_ptr(grad_flat),
                                                       *(_ptr(t) for t in self.inputs),
                                                       *self._common(), self.image_elems,
                                                       self.mpr, _ptr(gE),
                                                       _ptr(gx), _ptr(gM), _ptr(self.ws),
                                                       self.ws.numel(), ctypes.byref(self.cfg),
                                                       _stream(self.device)))
        return None if records else (gE, gx, gM)

    def images(self, flat):
        return [flat[o:o + C * H * W].view(C, H, W)
                for o, (C, H, W) in zip(self.offsets, self.shapes)]
