"""Analytic depth peeling on one NVIDIA B200 (sm_100a), behind the reference's
``warp_peel`` call surface: ``DevicePeeler``, ``EventPeeler``,
``Capacities``, ``EventCapacities`` (warp_peel/__init__.py:3-6)."""

from .events import EventCapacities, EventPeeler
from .solver import Capacities, DevicePeeler

__all__ = ["Capacities", "DevicePeeler", "EventCapacities", "EventPeeler"]
