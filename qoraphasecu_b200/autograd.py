"""Differentiable amplitude loss for gradient-based reconstruction.

``AmplitudeLoss`` is a ``torch.autograd.Function`` whose forward and backward
run the hand-written loss/adjoint line passes of libqpb.so
(``qpb_amplitude_loss_grad``): for each object x_b of a batch,

    L_b(x) = sum over usable pixels of (|F x_b| - A)^2,     F the unitary FFT,
    dL_b/dRe x + i dL_b/dIm x = 2 F^H[(|y| - A) y / |y|] = 2 (x_b - P_M x_b),

P_M being the reference's modulus projection. The gradient is computed in
the forward call and kept for backward. Objects live in FFT order on the
device (``to_fft_order`` / ``to_centred`` convert); PyTorch only holds the
memory and runs the optimiser step.

``adam_reconstruct`` is the gradient-based counterpart of ``reconstruct``:
random starts drawn exactly as the projection solver draws them, Adam on the
amplitude loss, and after every step the projection onto the support and onto
a per-pixel magnitude bound.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _lib
from .api import Problem, Reconstruction, Solver


def _torch():
    import torch

    return torch


class AmplitudeModel:
    """The problem's signed amplitude (-1 on masked pixels) and support, FFT order, on a device."""

    def __init__(self, problem: Problem, device: str = "cuda"):
        torch = _torch()
        amp = np.fft.ifftshift(problem.amplitude).astype(np.float32)
        mask = np.fft.ifftshift(problem.mask)
        signed = np.where(mask != 0, np.float32(-1.0), amp).astype(np.float32)
        self.shape = tuple(problem.shape)
        self.signed = torch.from_numpy(np.ascontiguousarray(signed)).to(device)
        self.support = torch.from_numpy(
            np.ascontiguousarray(np.fft.ifftshift(problem.support) != 0)).to(device)
        self.energy = float(np.sum(np.where(mask != 0, 0.0, amp.astype(np.float64) ** 2)))

    def scaled(self, scale: float) -> "AmplitudeModel":
        """The model of objects measured in units of ``scale``: the amplitude
        divided by it (masked pixels stay -1) and the energy by its square,
        so that the loss of x / scale is the loss of x divided by scale^2."""
        out = object.__new__(AmplitudeModel)
        out.shape = self.shape
        out.support = self.support
        out.signed = _divide_usable(self.signed, scale)
        out.energy = self.energy / (scale * scale)
        return out


def _divide_usable(signed, scale):
    """The signed amplitude divided by ``scale`` on usable pixels (>= 0), -1 kept on masked ones."""
    torch = _torch()
    return torch.where(signed >= 0, signed / scale, signed).contiguous()


def _loss_and_grad(x, signed, shape):
    torch = _torch()
    if not x.is_cuda or x.dtype != torch.complex64:
        raise ValueError("x must be a complex64 CUDA tensor")
    x = x.contiguous()
    batch = x.numel() // int(np.prod(shape))
    if batch * int(np.prod(shape)) != x.numel():
        raise ValueError(f"x of {x.numel()} elements is not a batch of {shape}")
    grad = torch.empty_like(x)
    loss = torch.empty(batch, dtype=torch.float64, device=x.device)
    lib = _lib.load()
    stream = torch.cuda.current_stream(x.device).cuda_stream
    _lib.check(lib.qpb_amplitude_loss_grad(
        len(shape), _lib.shape_arg(shape), batch, ctypes.c_void_p(signed.data_ptr()),
        ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(grad.data_ptr()),
        ctypes.c_void_p(loss.data_ptr()), ctypes.c_void_p(stream)))
    return loss, grad


def project_support_bound(x, support, bound=None):
    """In place on FFT-order objects x (complex64 CUDA tensor (..., *shape)):
    0 outside ``support`` (bool CUDA tensor of the objects' shape), and inside
    it every magnitude above ``bound`` scaled down onto ``bound`` (None: the
    support alone). One pass of libqpb.so (``qpb_project_support_bound``) on
    the current stream. Returns x."""
    torch = _torch()
    if not x.is_cuda or x.dtype != torch.complex64 or not x.is_contiguous():
        raise ValueError("x must be a contiguous complex64 CUDA tensor")
    if support.dtype != torch.bool or support.device != x.device or not support.is_contiguous():
        raise ValueError("support must be a contiguous bool tensor on x's device")
    numel = support.numel()
    if tuple(x.shape[x.dim() - support.dim():]) != tuple(support.shape):
        raise ValueError(f"x.shape {tuple(x.shape)} does not end with {tuple(support.shape)}")
    lib = _lib.load()
    stream = torch.cuda.current_stream(x.device).cuda_stream
    _lib.check(lib.qpb_project_support_bound(
        numel, x.numel() // numel, ctypes.c_void_p(support.data_ptr()),
        float("inf") if bound is None else float(bound), ctypes.c_void_p(x.data_ptr()),
        ctypes.c_void_p(stream)))
    return x


class AmplitudeLoss:
    """``AmplitudeLoss.apply(x, model)`` -> per-object losses (float64, shape (batch,))."""

    _function = None

    @classmethod
    def function(cls):
        if cls._function is None:
            torch = _torch()

            class _Fn(torch.autograd.Function):
                @staticmethod
                def forward(ctx, x, signed, shape):
                    loss, grad = _loss_and_grad(x, signed, shape)
                    ctx.save_for_backward(grad)
                    ctx.ndim = len(shape)
                    return loss

                @staticmethod
                def backward(ctx, g):
                    (grad,) = ctx.saved_tensors
                    scale = g.to(torch.float32).reshape(-1, *([1] * ctx.ndim))
                    return grad * scale, None, None

            cls._function = _Fn
        return cls._function

    @classmethod
    def apply(cls, x, model: AmplitudeModel):
        batch_shape = x.shape[: x.dim() - len(model.shape)]
        if tuple(x.shape[x.dim() - len(model.shape):]) != model.shape:
            raise ValueError(f"x.shape {tuple(x.shape)} does not end with {model.shape}")
        losses = cls.function().apply(x, model.signed, model.shape)
        return losses.reshape(batch_shape) if batch_shape else losses.reshape(())


def amplitude_loss(x, model: AmplitudeModel):
    """Per-object amplitude losses of FFT-order objects x (..., *shape)."""
    return AmplitudeLoss.apply(x, model)


def to_fft_order(x, ndim):
    """Centre-origin -> FFT order over the last ``ndim`` axes (torch tensors)."""
    torch = _torch()
    return torch.fft.ifftshift(x, dim=tuple(range(-ndim, 0)))


def to_centred(x, ndim):
    """FFT order -> centre-origin over the last ``ndim`` axes (torch tensors)."""
    torch = _torch()
    return torch.fft.fftshift(x, dim=tuple(range(-ndim, 0)))


def adam_reconstruct(problem: Problem, *, starts: int = 1, steps: int = 500, lr: float = 1e-2,
                     seed: int | None = None, init=None, seconds: float | None = None,
                     bound: float | None = 16.0, graph: bool = True, device: str = "cuda"):
    """Gradient-based reconstruction: Adam on the amplitude loss with the
    support projection after every step. Starts are drawn as ``Solver`` draws
    them (same seed -> same starting objects). Stops after ``steps`` steps or
    ``seconds`` of wall time, whichever comes first. Returns one
    ``Reconstruction`` per start; ``errors`` holds the Fourier error
    sqrt(L / energy) of every step, the projection solvers' error measure.

    Adam's step is absolute in the units of its parameters, and measured
    intensities fix the object's scale (counts), so the parameters are the
    object divided by the root-mean-square amplitude that a support of this
    size needs to carry the measured energy: ``lr`` is a step relative to the
    object's typical amplitude, whatever the photon count.

    The loss does not see the Fourier components under a beamstop mask, so
    nothing in it holds back the object along those directions, and Adam's
    per-pixel normalised steps let them grow without limit (on a 512^2 square
    with a beamstop of radius 12, pixels reached 700 times the RMS amplitude).
    ``bound`` caps every pixel's magnitude at ``bound`` times that RMS
    amplitude after each step (the projection onto a disc per pixel, which,
    like the support projection, leaves objects inside it unchanged); None
    turns the cap off.

    With ``graph`` (the default) the first three steps run eagerly (on a side
    stream, which also builds the optimiser's state and the library's plans)
    and one step is then captured as a CUDA graph and replayed for the rest:
    a step is about twenty small kernels whose launches from Python would
    otherwise take longer than the work. The arithmetic is the same either
    way (the fused Adam with ``capturable=True`` in both), so the objects are
    identical; only the FP64 sums of the per-step losses may differ in their
    last bits."""
    torch = _torch()
    with Solver(problem, starts=starts, seed=seed, init=init) as drawn:
        first = drawn.results()
    model = AmplitudeModel(problem, device)
    ndim = len(model.shape)
    x0 = np.stack([np.fft.ifftshift(r.object) for r in first]).astype(np.complex64)
    inside = max(int(model.support.sum().item()), 1)
    scale = float(np.sqrt(model.energy / inside)) or 1.0
    # Adam's parameter is the objects' real view (real and imaginary parts as
    # pairs), which is how torch's Adam treats a complex parameter; on the
    # real view it runs the fused implementation, one kernel per step instead
    # of about ten element-wise passes.
    w = torch.view_as_real(torch.from_numpy(x0 / np.float32(scale)).to(device)).clone()
    w.requires_grad_(True)
    support = model.support.contiguous()
    opt = torch.optim.Adam([w], lr=lr, capturable=True, fused=True)

    # The loss of the objects x = w scale is scale^2 times the loss of w
    # against the amplitude divided by scale: the passes run on w directly
    # (no scaled copy of the objects forward, nor of the gradient backward).
    model_w = model.scaled(scale)
    squared = scale * scale

    def one_step():
        losses = amplitude_loss(torch.view_as_complex(w), model_w) * squared
        losses.sum().backward()
        opt.step()
        with torch.no_grad():
            project_support_bound(torch.view_as_complex(w), support, bound)
        return losses.detach()

    def out_of_time():
        return seconds is not None and time.perf_counter() - t0 >= seconds

    history = []
    t0 = time.perf_counter()
    eager = min(steps, 3) if graph else steps
    side = torch.cuda.Stream(device=w.device)
    side.wait_stream(torch.cuda.current_stream(w.device))
    with torch.cuda.stream(side):
        for _ in range(eager):
            opt.zero_grad(set_to_none=True)
            history.append(one_step())
            if out_of_time():
                break
    torch.cuda.current_stream(w.device).wait_stream(side)
    if len(history) < steps and not out_of_time():
        captured = torch.cuda.CUDAGraph()
        opt.zero_grad(set_to_none=True)
        with torch.cuda.graph(captured):
            static_losses = one_step()
        while len(history) < steps and not out_of_time():
            captured.replay()
            history.append(static_losses.clone())
        del captured
    torch.cuda.synchronize()
    errors = torch.sqrt(torch.stack(history) / (model.energy + 1e-12)).to(torch.float32).cpu().numpy()
    final = to_centred(torch.view_as_complex(w.detach()) * scale, ndim).cpu().numpy()
    supp = np.fft.fftshift(model.support.cpu().numpy(), axes=tuple(range(-ndim, 0)))
    return [Reconstruction(final[s], supp.copy(), errors[:, s].copy()) for s in range(starts)]
