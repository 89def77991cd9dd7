"""Build step for the oracle pins (TEST INFRASTRUCTURE ONLY).

Reads two of the reference's solver sources where they lie in its tree and writes the
definitions the pins need to ``oracle/_ref/solver_extract.inc`` (git-ignored; nothing of
the reference is committed):

* ``src/solver/contact_solver.cu``: the float3 helpers (operators, dot, fnorm, ele,
  load_float3) and the kernels ``compute_Scc_kernel`` (S_c, Gamma_c, K_c),
  ``update_p_kernel`` (warm start p += Gamma r_c), ``get_delta_u_kernel`` (friction-cone
  projection) and ``update_p`` (per-vertex gather of the projection);
* ``src/solver/jacobi_solver.cu``: ``struct JacobiFunctor`` (one Jacobi row).

Definitions are found by their signatures and cut at their matching closing brace, so the
recipe does not depend on line numbers.  ``oracle/ref_pin_solver.cpp`` includes the result
between host stand-ins for the CUDA built-ins and runs each kernel serially.

    python oracle/ref_extract.py <reference root> <output .inc>
"""
import re
import sys


def cut(src: str, start: int) -> int:
    """End (exclusive) of the brace block that opens at or after `start`, plus a trailing ';'."""
    i = src.index("{", start)
    depth = 0
    while True:
        ch = src[i]
        if ch == "{":
            depth += 1
        elif ch == "}":
            depth -= 1
            if depth == 0:
                i += 1
                break
        i += 1
    j = i
    while j < len(src) and src[j] in " \t":
        j += 1
    if j < len(src) and src[j] == ";":
        i = j + 1
    return i


def definition(src: str, pattern: str) -> str:
    m = re.search(pattern, src, re.M)
    if not m:
        raise SystemExit(f"definition not found: {pattern}")
    return src[m.start():cut(src, m.end())]


def main(root: str, out: str) -> None:
    cs = open(f"{root}/src/solver/contact_solver.cu").read()
    js = open(f"{root}/src/solver/jacobi_solver.cu").read()
    # the helper block: from the first float3 operator up to the first device atomic helper
    a = re.search(r"^__host__ __device__ inline float3 operator\+", cs, re.M)
    b = re.search(r"^__device__ inline void atomicAdd_F3", cs, re.M)
    if not a or not b or b.start() <= a.start():
        raise SystemExit("helper block of contact_solver.cu not found")
    parts = [
        "// extracted by oracle/ref_extract.py from src/solver/contact_solver.cu",
        cs[a.start():b.start()],
        definition(cs, r"^__global__ void compute_Scc_kernel\("),
        definition(cs, r"^__global__ void update_p_kernel\("),
        definition(cs, r"^__global__ void get_delta_u_kernel\("),
        definition(cs, r"^__global__ void update_p\("),
        "// extracted by oracle/ref_extract.py from src/solver/jacobi_solver.cu",
        definition(js, r"^struct JacobiFunctor\s*"),
    ]
    with open(out, "w") as f:
        f.write("\n\n".join(parts) + "\n")


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
