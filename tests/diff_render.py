"""torch.autograd wrapper of the renderer's forward pass (pt_render with fixed
spp) and its path-replay adjoint (pt_backward), for tests that optimise
material parameters.  Test infrastructure: the product API is PathTracer."""
import numpy as np
import torch

PARAMS = ("r", "g", "b", "roughness", "metallic", "sheen", "emission")


def apply_theta(base: np.ndarray, theta: np.ndarray) -> np.ndarray:
    """Materials with the 7 differentiable fields of each row replaced by theta."""
    m = base.copy()
    for j, name in enumerate(PARAMS):
        m[name] = theta[:, j].astype(np.float32)
    return m


def theta_of(materials: np.ndarray) -> np.ndarray:
    return np.stack([materials[name].astype(np.float64) for name in PARAMS], -1)


class RenderImage(torch.autograd.Function):
    """image = render(theta); d loss / d theta by pt_backward."""

    @staticmethod
    def forward(ctx, theta, tracer, base_materials, spp):
        mats = apply_theta(base_materials, theta.detach().cpu().numpy())
        tracer.set_materials(mats)
        tracer.reset_accumulation()
        tracer.render(spp)
        rgba, counts, _ = tracer.readback()
        assert np.all(counts == spp)
        ctx.tracer, ctx.spp, ctx.m = tracer, spp, theta.shape[0]
        return torch.from_numpy(rgba[..., :3].astype(np.float32).copy())

    @staticmethod
    def backward(ctx, grad_img):
        g, _ = ctx.tracer.backward(grad_img.detach().cpu().numpy().astype(np.float32), ctx.spp)
        return torch.from_numpy(g[:ctx.m].astype(np.float64)), None, None, None
