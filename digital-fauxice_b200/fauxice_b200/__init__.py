"""B200 backend for the Digital ICE processing core of portable_digital_ice.

Public entry points mirror the reference package: ``process(job,
backend="b200")``, ``process_b200`` (the backend function, like
``process_cuda``), ``b200_self_test``, and ``run_streaming_replay_b200``
(like ``run_streaming_replay``).  The compute path is libfauxice_b200.so
(CUDA for sm_100a) through ctypes; nothing here computes pixels on the CPU.
"""

from .backend import (BackendProcessingResult, BackendSelection, ComputeBackend, b200_self_test,
                      process, synthetic_self_test_job)
from .contracts import (AcquisitionEpoch, DualRGBIAcquisition, PrepassFrameRecord, ProcessingJob,
                        ProcessingMode, RGBI16Frame, ScannerModel)
from .engine import (B200BackendUnavailable, ProcessingCancelled, ProcessingDiagnostics,
                     ProcessingPhase, ProcessingProgress, ProcessingResult, StartupReplayResult,
                     StreamingReplayResult, process_b200)
from .profile import DEFAULT_PROFILE, LS5000Selector8NormalProfile
from .streaming import run_streaming_replay_b200

__version__ = "0.1.0"

__all__ = [
    "AcquisitionEpoch",
    "B200BackendUnavailable",
    "BackendProcessingResult",
    "BackendSelection",
    "ComputeBackend",
    "DEFAULT_PROFILE",
    "DualRGBIAcquisition",
    "LS5000Selector8NormalProfile",
    "PrepassFrameRecord",
    "ProcessingCancelled",
    "ProcessingDiagnostics",
    "ProcessingJob",
    "ProcessingMode",
    "ProcessingPhase",
    "ProcessingProgress",
    "ProcessingResult",
    "RGBI16Frame",
    "ScannerModel",
    "StartupReplayResult",
    "StreamingReplayResult",
    "b200_self_test",
    "process",
    "process_b200",
    "run_streaming_replay_b200",
    "synthetic_self_test_job",
]
