#!/usr/bin/env python3
"""Generate the golden fixtures in this folder from the reference's own code.

Run in a container that has the reference checkout (read-only is fine):

    python tests/golden/gen_golden.py --reference /path/to/reference

The reference's kernels need NVIDIA Warp, which is not installed there, so the
fixtures come from the parts of the reference that run without it:

* ``pfflip/config.py`` and ``pfflip/scenes.py`` (pure NumPy), loaded by file
  path into a stand-in package: seeded particle positions/types (bit-exact
  seeding pins).
* ``random_beta`` and ``assemble`` from ``tests/test_poisson.py:23-78``
  (NumPy/SciPy), extracted with ``ast`` because that module imports ``warp`` at
  its top: the assembled-matrix product of ``test_operator_matches_assembled``
  (``tests/test_poisson.py:88-111``) and the ``spsolve`` solution of
  ``test_mgpcg_solves`` (``tests/test_poisson.py:114-145``), on the same seeds.
* ``Simulator._calibrate_rho_tilde_0`` (``pfflip/sim.py:119-140``), extracted the
  same way: ρ̃₀ for several (dx, ppc).

Outputs: ``golden.npz`` (arrays) and ``golden.json`` (scalars, hashes).
"""

from __future__ import annotations

import argparse
import ast
import hashlib
import importlib.util
import json
import os
import sys
import types

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

HERE = os.path.dirname(os.path.abspath(__file__))


def load_ref_package(ref):
    """Load pfflip/config.py and pfflip/scenes.py under a stand-in package name."""
    pkg = types.ModuleType("_refpf")
    pkg.__path__ = [os.path.join(ref, "pfflip")]
    sys.modules["_refpf"] = pkg
    mods = {}
    for name in ("config", "scenes"):
        spec = importlib.util.spec_from_file_location(f"_refpf.{name}", os.path.join(ref, "pfflip", f"{name}.py"))
        m = importlib.util.module_from_spec(spec)
        sys.modules[f"_refpf.{name}"] = m
        spec.loader.exec_module(m)
        mods[name] = m
    return mods["config"], mods["scenes"]


def extract_functions(path, names, extra_globals=None):
    """exec only the named top-level function definitions of a source file."""
    src = open(path).read()
    tree = ast.parse(src)
    g = {"np": np, "sp": sp, "spla": spla, "math": __import__("math")}
    if extra_globals:
        g.update(extra_globals)
    for node in tree.body:
        if isinstance(node, ast.FunctionDef) and node.name in names:
            exec(compile(ast.Module([node], []), path, "exec"), g)
    return {n: g[n] for n in names}


def extract_method(path, cls, meth):
    src = open(path).read()
    tree = ast.parse(src)
    for node in tree.body:
        if isinstance(node, ast.ClassDef) and node.name == cls:
            for item in node.body:
                if isinstance(item, ast.FunctionDef) and item.name == meth:
                    g = {"math": __import__("math"), "np": np}
                    exec(compile(ast.Module([item], []), path, "exec"), g)
                    return g[meth]
    raise KeyError(meth)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True)
    args = ap.parse_args()
    ref = args.reference
    config, scenes = load_ref_package(ref)
    Config = config.Config
    arrays, meta = {}, {}

    # ---- seeding pins (pfflip/scenes.py:17-169) -------------------------
    seeds = {
        "dam_break_8_ppc8": (lambda c: scenes.dam_break(c), dict(res=(8, 8, 8), dx=1 / 8, ppc=8)),
        "dam_break_6_ppc27": (lambda c: scenes.dam_break(c), dict(res=(6, 6, 6), dx=1 / 6, ppc=27)),
        "still_pool_10x8x6": (lambda c: scenes.still_pool(c, fill=0.5), dict(res=(10, 8, 6), dx=0.1, ppc=8)),
        "asteroid_12": (lambda c: scenes.asteroid_impact(c), dict(res=(12, 12, 12), dx=1 / 12, ppc=8)),
        "rayleigh_taylor_8": (lambda c: scenes.rayleigh_taylor(c), dict(res=(8, 8, 8), dx=1 / 8, ppc=8)),
    }
    for key, (fn, kw) in seeds.items():
        cfg = Config(**kw, seed=42)
        pos, vel, pt = fn(cfg)
        arrays[f"seed_{key}_pos"] = pos
        arrays[f"seed_{key}_vel"] = vel
        arrays[f"seed_{key}_ptype"] = pt
    cfg = Config(res=(16, 16, 16), dx=1 / 16, ppc=8, seed=42)
    pos, vel, pt, solid = scenes.wave_vs_tower(cfg)
    arrays["seed_wave_vs_tower_16_pos"] = pos
    arrays["seed_wave_vs_tower_16_vel"] = vel
    arrays["seed_wave_vs_tower_16_ptype"] = pt
    arrays["seed_wave_vs_tower_16_solid"] = solid
    # hash pin of the 32^3 / 8 ppc dam break (262,144 particles)
    cfg = Config(res=(32, 32, 32), dx=1 / 32, ppc=8, seed=42)
    pos, vel, pt = scenes.dam_break(cfg)
    meta["dam_break_32_ppc8"] = {"n": int(len(pos)), "n_liquid": int((pt == 1).sum()),
                                 "sha_pos": sha(pos), "sha_ptype": sha(pt)}

    # ---- operator and solver pins (tests/test_poisson.py) ---------------
    tp = os.path.join(ref, "tests", "test_poisson.py")
    fns = extract_functions(tp, ["random_beta", "assemble"])
    random_beta, assemble = fns["random_beta"], fns["assemble"]
    RES = (16, 16, 16)
    for contrast in (1.0, 1000.0):
        tag = f"c{int(contrast)}"
        rng = np.random.default_rng(0)
        bx, by, bz = random_beta(RES, rng, contrast)
        A = assemble(RES, bx, by, bz)
        p = rng.random(RES).astype(np.float32)
        Ap = (A @ p.astype(np.float64).ravel()).reshape(RES)
        arrays[f"op_{tag}_bx"], arrays[f"op_{tag}_by"], arrays[f"op_{tag}_bz"] = bx, by, bz
        arrays[f"op_{tag}_p"], arrays[f"op_{tag}_Ap"] = p, Ap
        meta[f"op_{tag}_sym"] = float(abs(A - A.T).max())
        meta[f"op_{tag}_rowsum"] = float(np.abs(np.asarray(A.sum(axis=1)).ravel()).max())

        rng = np.random.default_rng(1)
        bx, by, bz = random_beta(RES, rng, contrast)
        A = assemble(RES, bx, by, bz)
        b = rng.standard_normal(RES).astype(np.float64)
        b -= b.mean()
        n = A.shape[0]
        sol = spla.spsolve((A + sp.eye(n) * 1e-10).tocsc(), b.ravel())
        sol -= sol.mean()
        arrays[f"solve_{tag}_bx"], arrays[f"solve_{tag}_by"], arrays[f"solve_{tag}_bz"] = bx, by, bz
        arrays[f"solve_{tag}_b"] = b.astype(np.float32)
        arrays[f"solve_{tag}_x"] = sol.reshape(RES)

    # ---- rho~_0 (pfflip/sim.py:119-140) ---------------------------------
    calib = extract_method(os.path.join(ref, "pfflip", "sim.py"), "Simulator", "_calibrate_rho_tilde_0")
    rt = {}
    for dx, ppc in ((1 / 8, 8), (1 / 16, 8), (1 / 16, 27), (1 / 24, 8), (1 / 32, 8), (1 / 64, 8), (1 / 128, 27)):
        fake = types.SimpleNamespace(cfg=Config(res=(8, 8, 8), dx=dx, ppc=ppc))
        rt[f"{dx!r}_{ppc}"] = calib(fake)
    meta["rho_tilde_0"] = rt

    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", len(arrays), "arrays and", len(meta), "meta entries")


if __name__ == "__main__":
    main()
