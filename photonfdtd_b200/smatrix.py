"""Modal amplitudes and S-parameters at a waveguide port: the counterpart of
the reference's smatrix module (src/photonfdtd/smatrix.py:41-118), same
functions and arguments.

A port is a plane normal to x carrying DFT fields Ey, Ez, Hy, Hz (a
plane-restricted DFTMonitor). The amplitude of a mode in the simulated field
is the ratio of two reciprocity overlaps,
    <a, b> = sum over the plane of (conj(E_a) x H_b + E_b x conj(H_a)) . x dA,
alpha+ = <m+, sim> / <m+, m+> for the mode as solved and alpha- with its
transverse H reversed (the backward mode, orthogonal to the forward one
under this product). Only element-wise products, conj, reshape and a sum
over the last axis are used, so the functions take NumPy arrays or torch
tensors alike: CUDA tensors keep the overlaps on the device, and tensors
that require grad (the ``out['dft']`` leaves of
``photonfdtd_b200.adjoint.value_and_grad_eps``) make |S|^2 a differentiable
loss, the mode held fixed.
"""
from __future__ import annotations

from typing import Dict, Tuple

import numpy as np

PORT_COMPONENTS = ("Ey", "Ez", "Hy", "Hz")


def _overlap(a, b, dA):
    """<a, b> for 4-tuples (Ey, Ez, Hy, Hz) flattened over the plane (the
    last axis), with an optional leading frequency axis."""
    ey_a, ez_a, hy_a, hz_a = a
    ey_b, ez_b, hy_b, hz_b = b
    s = (ey_a.conj() * hz_b - ez_a.conj() * hy_b) + (ey_b * hz_a.conj() - ez_b * hy_a.conj())
    return s.sum(-1) * dA


def mode_amplitudes(sim_fields: Dict, mode_fields: Dict, dA: float):
    """(alpha_plus, alpha_minus) per frequency: ``sim_fields`` maps Ey, Ez,
    Hy, Hz to (n_freq, ...) port arrays, ``mode_fields`` the mode's four
    components on the same transverse cells, ``dA`` the cell area."""
    sim = tuple(sim_fields[c].reshape(sim_fields[c].shape[0], -1) for c in PORT_COMPONENTS)
    ey, ez, hy, hz = (mode_fields[c].reshape(-1) for c in PORT_COMPONENTS)
    fwd, bwd = (ey, ez, hy, hz), (ey, ez, -hy, -hz)
    return (_overlap(fwd, sim, dA) / _overlap(fwd, fwd, dA),
            _overlap(bwd, sim, dA) / _overlap(bwd, bwd, dA))


def port_fields(result, monitor_name: str) -> Dict:
    """The four tangential DFT components of a port monitor of a Result (or
    of the ``out['dft']`` dict of a loss)."""
    dft = result.dft[monitor_name] if hasattr(result, "dft") else result["dft"][monitor_name]
    missing = [c for c in PORT_COMPONENTS if c not in dft]
    if missing:
        raise ValueError(f"port monitor {monitor_name!r} is missing components {missing}; "
                         f"record components={PORT_COMPONENTS} on the port plane")
    return {c: dft[c] for c in PORT_COMPONENTS}


def mode_port_fields(mode_result, mode_index: int = 0, like=None) -> Dict:
    """The four tangential components of mode ``mode_index``; with ``like``
    (a torch tensor) as tensors of its device."""
    out = {c: np.asarray(getattr(mode_result, c)[mode_index]) for c in PORT_COMPONENTS}
    if like is not None and not isinstance(like, np.ndarray):
        import torch
        out = {c: torch.as_tensor(v, dtype=torch.complex128, device=like.device)
               for c, v in out.items()}
    return out


def s_parameters(result, out_monitor: str, mode_result, mode_index: int = 0,
                 dA: float = 1.0) -> Tuple:
    """(alpha_plus, alpha_minus) of mode ``mode_index`` at the port monitor
    ``out_monitor`` over its frequencies; with a unit-power one-way source at
    another port, alpha_plus is the S-parameter into this port."""
    sim = port_fields(result, out_monitor)
    return mode_amplitudes(sim, mode_port_fields(mode_result, mode_index, like=sim["Ey"]), dA)
