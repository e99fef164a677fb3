"""B200-native unsplit hydro block update with FLASH5's Hydro interface.

The hot path lives in the CUDA library ``_flash_hy.so`` (C ABI declared in
include/flash_hy.h); ``flash5_b200.hydro.Hydro`` is the host-side mirror of
the reference's Hydro / Hydro_computeDt calls.
"""
