"""Prepares bismit's OpenCL kernel sources for compilation as C++ (TEST INFRASTRUCTURE).

Reads cl/bismit.cl, cl/syns.cl, cl/control.cl, cl/filters.cl and cl/tests.cl
from a bismit
checkout and writes their concatenation to an output file (under oracle/_ref/,
never committed), changing exactly one construct: OpenCL vector literals
``(int4)(a, b, c, d)`` become C++ constructor calls ``int4(a, b, c, d)``. In
C++ the original spelling would be a cast of a comma expression. Casts of a
single scalar, such as ``(int4)0`` or ``(int4)(int)v``, already mean "splat"
in both languages and are left alone. The kernel code is otherwise unchanged.

Usage: python prep_cl.py <bismit checkout> <output file>
"""
import re
import sys

FILES = ["cl/bismit.cl", "cl/syns.cl", "cl/control.cl", "cl/filters.cl", "cl/tests.cl"]
VEC_CAST = re.compile(r"\((u?char4|u?short4|u?int4)\)\s*\(")


def _matching_paren(s, i):
    depth = 0
    for j in range(i, len(s)):
        if s[j] == "(":
            depth += 1
        elif s[j] == ")":
            depth -= 1
            if depth == 0:
                return j
    raise ValueError("unbalanced parentheses at %d" % i)


def _has_top_level_comma(s):
    depth = 0
    for ch in s:
        if ch in "([":
            depth += 1
        elif ch in ")]":
            depth -= 1
        elif ch == "," and depth == 0:
            return True
    return False


def rewrite_vector_literals(src):
    out = []
    pos = 0
    while True:
        m = VEC_CAST.search(src, pos)
        if not m:
            out.append(src[pos:])
            break
        open_i = m.end() - 1
        close_i = _matching_paren(src, open_i)
        inner = src[open_i + 1:close_i]
        if _has_top_level_comma(inner):
            out.append(src[pos:m.start()])
            out.append("%s(%s)" % (m.group(1), rewrite_vector_literals(inner)))
            pos = close_i + 1
        else:
            out.append(src[pos:m.end()])
            pos = m.end()
    return "".join(out)


def main():
    root, dst = sys.argv[1], sys.argv[2]
    parts = []
    for f in FILES:
        with open("%s/%s" % (root, f)) as fh:
            parts.append("// ---- %s ----\n" % f)
            parts.append(rewrite_vector_literals(fh.read()))
            parts.append("\n")
    with open(dst, "w") as fh:
        fh.write("".join(parts))


if __name__ == "__main__":
    main()
