"""Exception types of the reference API (backends/base.py:15-16, checkpoint.py:28-29)."""


class BackendUnavailableError(RuntimeError):
    """Raised when a requested compute backend or device cannot be used."""


class CheckpointError(ValueError):
    """Raised when a checkpoint is unsupported, corrupt, or inconsistent."""
