"""cuwaves: B200 engine for the CP-PAW wavefunction hot path (host-side binding).

The compute path is the CUDA library lib/libcuwaves.so behind the C ABI of
include/cuwaves.h; this package only binds it (capi) and builds seeded model
inputs (systems).
"""
from . import systems  # noqa: F401
from .capi import (Batch, CUW_HPSI, CUW_OPSI, CUW_OPT_FFT_VARIANT, CUW_OPT_GRAPHS, CUW_OPT_LYAP_MAX_SWEEPS,  # noqa: F401
                   CUW_OPT_SAFEORTHO, CUW_OPT_SELFCONSISTENT, CUW_OPT_LYAP_TOL, CUW_OPT_STREAM_PRIORITY,  # noqa: F401
                   CUW_OPT_SWAPSTATES, CUW_OPT_CONTRACTION_TILES, CUW_OPT_SM_SHARE,  # noqa: F401
                   CUW_PREC_FP64, CUW_PREC_MIXED, CUW_PSI0, CUW_PSIM, Waves, WavesError, bind, engine,
                   load_library, open_waves)
