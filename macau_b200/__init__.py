"""B200 (sm_100a) Gibbs sampler for BPMF / Macau matrix factorization.

Drop-in for the hot path of jaak-s/macau: ``macau()``, ``bpmf()``, ``blockcg()``,
``make_train_test()``, ``make_train_test_df()`` and ``MacauResult`` mirror the reference's Python
API (python/macau/macau.pyx); the sweeps run in hand-written CUDA behind the C ABI of
include/macau_b200.h (``macau_b200._lib``).
"""
__version__ = "0.1.0"

from .macau import (MacauResult, blockcg, blockcg_solve, bpmf, macau, make_train_test,
                    make_train_test_df)

__all__ = ["macau", "bpmf", "blockcg", "blockcg_solve", "make_train_test", "make_train_test_df",
           "MacauResult", "__version__"]
