"""Double-precision twin of the reference solver (test infrastructure, not the product).

Copies the reference's core sources into an output folder with every single-precision
type, literal, function and limit turned into its double-precision counterpart, so that
the same algorithm runs in FP64. The reference checkout is only read. The rules:

  * the type: the word ``float`` becomes ``double`` (``float3``, ``float3x3`` keep their
    names; their members are declared ``float`` and so become ``double``);
  * literals: a decimal literal with an ``f`` suffix (``0.5f``, ``1e-5f``) loses the suffix;
  * maths: ``sqrtf fabsf cbrtf sinf cosf`` (and the other ``<cmath>`` f-suffixed names
    used) become ``sqrt fabs cbrt sin cos``;
  * limits: ``FLT_MAX`` becomes ``DBL_MAX``, ``FLT_EPSILON`` becomes ``DBL_EPSILON``.

Nothing else changes: the same expression trees, branches and constants (in double).

    python make_fp64.py <reference source folder> <output folder>
"""
from __future__ import annotations

import os
import re
import sys

# the core files of the step (solver, narrowphase, forces, bodies, dense world) and the
# headers they include
FILES = ("solver.cpp", "collide.cpp", "manifold.cpp", "joint.cpp", "spring.cpp", "force.cpp", "rigid.cpp",
         "sim_world.cpp", "maths.h", "solver.h", "parallel_for.h")

_MATH = ("sqrt", "fabs", "cbrt", "sin", "cos", "tan", "atan2", "atan", "acos", "asin", "exp", "log", "pow",
         "floor", "ceil", "fmin", "fmax", "round", "fmod", "hypot", "copysign")
_RULES = [
    (re.compile(r"\bfloat\b"), "double"),
    (re.compile(r"\b((?:\d+\.\d*|\.\d+|\d+\.)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)[fF]\b"), r"\1"),
    (re.compile(r"\b(" + "|".join(_MATH) + r")f(?=\s*\()"), r"\1"),
    (re.compile(r"\bFLT_MAX\b"), "DBL_MAX"),
    (re.compile(r"\bFLT_EPSILON\b"), "DBL_EPSILON"),
    (re.compile(r"\bFLT_MIN\b"), "DBL_MIN"),
]


def to_fp64(text: str) -> str:
    for rx, rep in _RULES:
        text = rx.sub(rep, text)
    return text


def main(src: str, out: str) -> None:
    os.makedirs(out, exist_ok=True)
    for name in FILES:
        with open(os.path.join(src, name)) as f:
            text = f.read()
        dst = os.path.join(out, name)
        new = "// double-precision copy made by make_fp64.py; do not edit\n" + to_fp64(text)
        if os.path.exists(dst) and open(dst).read() == new:
            continue
        with open(dst, "w") as f:
            f.write(new)


if __name__ == "__main__":
    if len(sys.argv) != 3:
        sys.exit(__doc__)
    main(sys.argv[1], sys.argv[2])
