"""B200-native whole-brain LIF engine behind the reference's ``Brain`` / ``BatchBrain`` API.

Modules mirror the reference's names: ``brain`` (``LIFParams``, ``Brain``), ``gpu``
(``BatchBrain``), ``learning`` / ``batch`` (plastic-synapse rules), ``connectome`` (synthetic
stand-ins for FlyWire) and ``workloads`` (seeded benchmark inputs).
"""

from .brain import Brain, LIFParams  # noqa: F401


def __getattr__(name):
    if name == "BatchBrain":
        from .gpu import BatchBrain

        return BatchBrain
    raise AttributeError(name)
