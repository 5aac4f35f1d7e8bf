"""Second-quantized model container (``second_quantized_model.py:48-130`` of
the reference): a lattice plus 1-based bilinear ``(i, j, t)`` and density
``(i, j, V)`` term lists; the twisted-boundary update regenerates the
bilinear terms with Peierls phases."""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

from .lattice import generate_bilinear_terms
from .symmetry import Particle_Statistics

__all__ = [
    "Particle_Statistics",
    "Real_Space_Second_Quantized_Model",
    "update_second_quantized_model_with_twisted_phases",
]


@dataclass
class Real_Space_Second_Quantized_Model:
    params: dict[str, Any]
    lattice: Any
    tb_model: Any
    particle_statistics: Particle_Statistics
    bilinear_terms: list[tuple[int, int, complex]] = field(default_factory=list)
    density_density_terms: list[tuple[int, int, complex]] = field(default_factory=list)


def update_second_quantized_model_with_twisted_phases(
    second_quantized_model: Real_Space_Second_Quantized_Model,
    *,
    twisted_phases_over_2π: list[float],
) -> Real_Space_Second_Quantized_Model:
    """In place: bilinear terms with twisted phases, lattice flux recorded."""
    lattice = second_quantized_model.lattice
    if len(twisted_phases_over_2π) != lattice.dim:
        raise ValueError(f"twisted_phases_over_2π must have length {lattice.dim}.")
    second_quantized_model.bilinear_terms = generate_bilinear_terms(
        second_quantized_model.tb_model, twisted_phases_over_2π=twisted_phases_over_2π
    )
    lattice.twisted_phases_over_2π = list(twisted_phases_over_2π)
    return second_quantized_model
