"""B200-native optical-photon transport engine (drop-in for the GPU path of
zmeskma/GPU_Optical_photons).

The compute path is liboptx.so (hand-written CUDA for sm_100a behind the C ABI
of include/optx.h); this package is its Python binding: the reference-shaped
backend (``backend``), the wavefront / batched engine (``wavefront``) and the
differentiable tally (``adjoint``).
"""
from .params import (SimParams, TallyConfig, CSimParams, CFaces, CTallyConfig, INF,
                     POLISHED, BLACK, SPECULAR, LAMBERTIAN, POINT, VOLUME,
                     DETECTED, ABSORBED_BULK, ABSORBED_SURFACE, ESCAPED, MAX_STEPS, NUM_FATES,
                     FATE_NAMES, config1, config2, config3, black_box, default_cfg)
from ._lib import OptxError, InvalidArgument
from .backend import (Records, Tally, gpu_available, gpu_device_name, run_gpu_records,
                      run_gpu_tally, run_gpu_records_event, records_device, tally_device,
                      device_records, records_to_numpy)
from .wavefront import (EventTable, SortedEngine, WavefrontEngine, WaveConfig, wavefront_tally,
                        batched_events)


def __getattr__(name):
    # The differentiable response needs torch; import it on first use.
    if name in ("ResponseModel", "response", "loss_fn", "nll_loss", "calibrate", "crn_central_fd",
                "target_histogram"):
        from . import adjoint
        return getattr(adjoint, name)
    raise AttributeError(name)

__all__ = [n for n in dir() if not n.startswith("_")]
