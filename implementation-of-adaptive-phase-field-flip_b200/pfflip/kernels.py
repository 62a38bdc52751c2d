"""Launch shim for reference-style kernel calls.

Reference tests launch kernels directly, e.g.
``wp.launch(apply_A, dim=RES, inputs=[p, bx, by, bz, diag, out], device=DEV)``
(tests/test_poisson.py:106).  ``launch`` accepts the same call for the kernels
this package exposes as callables and forwards the inputs to them; the work
runs in libpfflip.so.
"""

from __future__ import annotations

from .poisson import apply_A  # noqa: F401


def launch(kernel, dim=None, inputs=(), device=None, **_ignored):
    """Run ``kernel(*inputs)``; ``dim`` and ``device`` are implied by the arrays."""
    if not callable(kernel):
        raise TypeError(f"{kernel!r} is not a launchable kernel of this package")
    return kernel(*inputs)
