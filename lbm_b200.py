"""Import name for the package in ``high-performance-lbm-on-gpu-_b200/``.

That directory name is not a Python identifier, so ``import lbm_b200`` loads it
through importlib; the package then registers itself and its submodules under
``lbm_b200``.
"""

import importlib
import sys

sys.modules[__name__] = importlib.import_module("high-performance-lbm-on-gpu-_b200")
