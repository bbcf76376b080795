"""hydist — B200-native ADI shallow-water + suspended-sediment step of GPU-hydist.

Python host side of the library: case parameters (:mod:`hydist.params`), synthetic
cases (:mod:`hydist.cases`), the ctypes binding of ``libhydist_b200.so``
(:mod:`hydist.lib`) and the Engine/rep-compatible calls (:mod:`hydist.engine`).
"""
from .params import HydCaseParams, default_params, derive  # noqa: F401
