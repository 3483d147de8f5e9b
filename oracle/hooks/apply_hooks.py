"""Writes a copy of KTPlace's globalPlacer/simpl/simpl_placer.cc whose
simplPlacer::Impl::getHpwl and ::getOccupancy call the B200 hooks
(ktplace_b200/dropin/simpl_hooks_b200.h) - the patch a maintainer would make
to route SimPL's HPWL and density passes to the GPU (simpl_placer.cc:256-289).

    python apply_hooks.py <reference simpl_placer.cc> <output file>

The two definitions are found by their signatures and their bodies replaced
(brace matching); the rest of the file is copied unchanged. Test
infrastructure: the oracle Makefile's `dropin` target builds the reference's
SimPL with it (oracle/_ref, never committed)."""
import os
import sys

BODIES = {
    "double simplPlacer::Impl::getHpwl(": """{
    return b200::hpwl(netlist, x, y);
}""",
    "std::vector<double> simplPlacer::Impl::getOccupancy(": """{
    return b200::occupancy(netlist, width, height, grid, densityLimit, x, y);
}""",
}
INCLUDE = '#include "simpl_hooks_b200.h"\n'


def replace_body(src: str, signature: str, body: str) -> str:
    i = src.find(signature)
    if i < 0 or src.find(signature, i + 1) >= 0:
        raise SystemExit(f"apply_hooks: expected one definition of {signature!r}")
    j = src.index("{", i)
    depth = 0
    for k in range(j, len(src)):
        if src[k] == "{":
            depth += 1
        elif src[k] == "}":
            depth -= 1
            if depth == 0:
                return src[:j] + body + src[k + 1:]
    raise SystemExit(f"apply_hooks: unbalanced braces after {signature!r}")


def main(argv) -> int:
    src = open(argv[1]).read()
    for sig, body in BODIES.items():
        src = replace_body(src, sig, body)
    first = src.index("#include")
    src = src[:first] + INCLUDE + src[first:]
    os.makedirs(os.path.dirname(argv[2]), exist_ok=True)
    open(argv[2], "w").write(src)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
