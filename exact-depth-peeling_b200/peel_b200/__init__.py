"""Analytic depth peeling on one NVIDIA B200 (sm_100a), behind the reference's
``warp_peel`` call surface: ``DevicePeeler``, ``EventPeeler``,
``Capacities``, ``EventCapacities`` (warp_peel/__init__.py:3-6)."""

from .batch import BatchPeeler
from .events import EventCapacities, EventPeeler
from .solver import Capacities, DevicePeeler

__all__ = ["BatchPeeler", "Capacities", "DevicePeeler", "EventCapacities", "EventPeeler"]
