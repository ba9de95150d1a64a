"""Drop-in ``MathUtils`` (reference: ``nep_simulator/MathUtils.py:3-24``)."""
import torch


def quaternion_multiplication(a, b):
    """Batched Hamilton product of (w, x, y, z) quaternions (not commutative):
    scalar a.s*b.s - dot(a.v, b.v), vector a.s*b.v + b.s*a.v + cross(a.v, b.v)."""
    res = torch.zeros_like(a)
    res[:, 0] = a[:, 0] * b[:, 0] - torch.sum(a[:, 1:] * b[:, 1:], dim=1)
    res[:, 1:] = a[:, :1] * b[:, 1:] + b[:, :1] * a[:, 1:] + torch.linalg.cross(a[:, 1:], b[:, 1:], dim=1)
    return res
