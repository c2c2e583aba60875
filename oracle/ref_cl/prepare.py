"""TEST INFRASTRUCTURE ONLY — prepares the reference's kernel source
(opencl/bmfr.cl) for the g++ build of oracle/_ref.

The kernels are compiled as C++ against `cl_compat.h`, which supplies the
OpenCL C surface they use (vector types and swizzles, built-in functions,
work-item functions, barriers).  Two constructs of OpenCL C have no C++
spelling a header can provide, so this script rewrites exactly those, line
for line (line numbers are kept, a `#line` directive names the source):

* a `__local`/`local` declaration *statement* inside a kernel
  (bmfr.cl:503, :659) declares one variable shared by the work-group; it
  becomes `CLC_KERNEL_LOCAL <declaration>` (a `static thread_local`: the
  executor runs a work-group's work-items as fibers of one thread).
  `__local` in parameter lists is left to the header (an empty macro);
* the component-wise vector select `v = v < 0.f ? 0.f : v;` (bmfr.cl:750)
  becomes `v = clc_vselect(v < 0.f, 0.f, v);`.

Every rule must match the expected number of times, otherwise the script
fails: a changed reference is never compiled silently.  The output goes to
oracle/_ref/ only; no reference source is kept in the repository.

Usage: python prepare.py <path of bmfr.cl> <output .inc>
"""
import re
import sys

RULES = [
    # (name, pattern, replacement, expected count)
    ("kernel-scope local declaration",
     re.compile(r"^(\s*)(?:__local|local)\s+([A-Za-z_]\w*\s+[A-Za-z_][^()]*;)\s*$"),
     r"\1CLC_KERNEL_LOCAL \2", 2),
    ("component-wise vector select",
     re.compile(r"^(\s*)(\w+) = (\w+) < 0\.f \? 0\.f : (\w+);\s*$"),
     r"\1\2 = clc_vselect(\3 < 0.f, 0.f, \4);", 1),
]


def prepare(src: str, name: str) -> str:
    lines = src.split("\n")
    counts = [0] * len(RULES)
    out = []
    for line in lines:
        for i, (_, pat, rep, _) in enumerate(RULES):
            new, n = pat.subn(rep, line)
            if n:
                counts[i] += n
                line = new
        out.append(line)
    for (rule, _, _, want), got in zip(RULES, counts):
        if got != want:
            raise SystemExit(f"prepare.py: rule '{rule}' matched {got} times, expected {want}")
    return f'#line 1 "{name}"\n' + "\n".join(out) + "\n"


def main():
    if len(sys.argv) != 3:
        raise SystemExit(__doc__)
    with open(sys.argv[1]) as f:
        src = f.read()
    text = prepare(src, "opencl/bmfr.cl")
    with open(sys.argv[2], "w") as f:
        f.write(text)


if __name__ == "__main__":
    main()
