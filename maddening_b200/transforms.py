"""Lattice <-> SI unit conversions for coupling edges.

Drop-in for MADDENING's ``src/maddening/core/transforms_unit.py:43-223``:
each factory fixes the physical scales and returns a pure function that
multiplies its argument by one constant, so it works unchanged on Python
floats, NumPy arrays and torch tensors (on any device, under autograd).
Names, argument order, the conversion factors and the ``__qualname__`` of the
returned function (used when a transform is registered by name) follow the
reference.

==========  ===========================================
quantity    multiply the lattice value by
==========  ===========================================
length      dx
velocity    dx / dt
force       rho dx^4 / dt^2   (si_to_lbm_force: inverse)
torque      rho dx^5 / dt^2
pressure    rho (dx / dt)^2
==========  ===========================================
"""

from __future__ import annotations


def _scale(factor: float, label: str):
    factor = float(factor)

    def _convert(x):
        return x * factor

    _convert.__qualname__ = label
    _convert.factor = factor
    return _convert


def lbm_to_si_force(dx_physical: float, dt_physical: float, rho_physical: float):
    """Lattice force -> newtons (transforms_unit.py:43-73)."""
    return _scale(rho_physical * dx_physical ** 4 / dt_physical ** 2,
                  f"lbm_to_si_force(dx={dx_physical}, dt={dt_physical}, rho={rho_physical})")


def si_to_lbm_force(dx_physical: float, dt_physical: float, rho_physical: float):
    """Newtons -> lattice force (transforms_unit.py:76-106)."""
    return _scale(dt_physical ** 2 / (rho_physical * dx_physical ** 4),
                  f"si_to_lbm_force(dx={dx_physical}, dt={dt_physical}, rho={rho_physical})")


def lbm_to_si_torque(dx_physical: float, dt_physical: float, rho_physical: float):
    """Lattice torque -> N m (transforms_unit.py:109-139)."""
    return _scale(rho_physical * dx_physical ** 5 / dt_physical ** 2,
                  f"lbm_to_si_torque(dx={dx_physical}, dt={dt_physical}, rho={rho_physical})")


def lbm_to_si_velocity(dx_physical: float, dt_physical: float):
    """Lattice velocity -> m/s (transforms_unit.py:142-168)."""
    return _scale(dx_physical / dt_physical,
                  f"lbm_to_si_velocity(dx={dx_physical}, dt={dt_physical})")


def lbm_to_si_pressure(dx_physical: float, dt_physical: float, rho_physical: float):
    """Lattice pressure -> pascals (transforms_unit.py:171-201)."""
    return _scale(rho_physical * (dx_physical / dt_physical) ** 2,
                  f"lbm_to_si_pressure(dx={dx_physical}, dt={dt_physical}, rho={rho_physical})")


def lbm_to_si_length(dx_physical: float):
    """Lattice length -> metres (transforms_unit.py:204-223)."""
    return _scale(dx_physical, f"lbm_to_si_length(dx={dx_physical})")


__all__ = ["lbm_to_si_force", "si_to_lbm_force", "lbm_to_si_torque", "lbm_to_si_velocity",
           "lbm_to_si_pressure", "lbm_to_si_length"]
