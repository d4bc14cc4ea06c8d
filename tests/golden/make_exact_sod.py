"""Generates tests/golden/exact_sod.npz from the reference's own exact Sod solver.

Imports exact_sod from the reference checkout's
share/spearhed/ValidationSetups/SodShockTube/validate_sod.py (its plotting
import, matplotlib, is not installed here and is not used by exact_sod, so a
bare stand-in module satisfies the import).  Run from the repository root:

    python tests/golden/make_exact_sod.py REFERENCE_ROOT

(REFERENCE_ROOT may also come from the REF_ROOT environment variable.)
"""
import importlib.util
import os
import sys
import types

import numpy as np

ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REF_ROOT")
if not ref_root:
    sys.exit("usage: make_exact_sod.py REFERENCE_ROOT (or set REF_ROOT): the reference checkout to import from")
path = os.path.join(ref_root, "share/spearhed/ValidationSetups/SodShockTube/validate_sod.py")
mpl = types.ModuleType("matplotlib")
mpl.use = lambda *a, **k: None
mpl.pyplot = types.ModuleType("matplotlib.pyplot")
sys.modules.setdefault("matplotlib", mpl)
sys.modules.setdefault("matplotlib.pyplot", mpl.pyplot)
spec = importlib.util.spec_from_file_location("validate_sod", path)
mod = importlib.util.module_from_spec(spec)
spec.loader.exec_module(mod)

x = np.linspace(-0.5 + 1e-6, 0.5 - 1e-6, 401)
out = {"x": x}
cases = [(0.05, 1.4), (0.1, 1.4), (0.2, 1.4), (0.1, 5.0 / 3.0), (0.1, 2.0)]
for k, (t, g) in enumerate(cases):
    rho, u, p, e = mod.exact_sod(x, t, gamma=g)
    out[f"t{k}"] = np.array([t, g])
    out[f"rho{k}"], out[f"u{k}"], out[f"p{k}"], out[f"e{k}"] = rho, u, p, e
dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "exact_sod.npz")
np.savez_compressed(dst, ncases=len(cases), **out)
print("wrote", dst)
