"""Patched copies of two reference sources for the 2D field-loop oracle.

The reference's induction solver advects with a hard-coded velocity
v = (1, 1, 0) (src/induction.cpp:29-31) and places its magnetic loop at
(0.5, 0.5) (src/initial_conditions.cpp:236-237). The 2D field-loop
configuration needs another velocity and centre, so this recipe writes
copies of those two files into the build folder (oracle/_ref/loop2d/,
git-ignored) with exactly those lines replaced by compile-time values
(SPDK_LOOP_VX, SPDK_LOOP_VY, SPDK_LOOP_CX, SPDK_LOOP_CY); nothing else
changes, and the copies are compiled with the other reference objects into
oracle/_ref/spd_K_loop2d (oracle/Makefile, target loop2d). Test
infrastructure only.

    python oracle/patch_loop2d.py <reference src dir> <output dir>
"""
import os
import sys


def patch(text, old, new, what):
    if text.count(old) != 1:
        raise SystemExit(f"patch_loop2d: the {what} text was not found exactly once")
    return text.replace(old, new)


def main(src, out):
    os.makedirs(out, exist_ok=True)
    with open(os.path.join(src, "induction.cpp")) as f:
        ind = f.read()
    ind = patch(ind, "double velocity(int var, double x, double y, double z){\n    if(var<2)return 1;\n    else return 0;",
                "double velocity(int var, double x, double y, double z){\n"
                "    return var==0 ? (double)(SPDK_LOOP_VX) : (var==1 ? (double)(SPDK_LOOP_VY) : 0.0);",
                "velocity()")
    with open(os.path.join(out, "induction.cpp"), "w") as f:
        f.write(ind)
    with open(os.path.join(src, "initial_conditions.cpp")) as f:
        ic = f.read()
    ic = patch(ic, "double magnetic_loop(int var, double x, double y, double z){\n    x = x-0.5;\n    y = y-0.5;",
               "double magnetic_loop(int var, double x, double y, double z){\n"
               "    x = x-(double)(SPDK_LOOP_CX);\n    y = y-(double)(SPDK_LOOP_CY);",
               "magnetic_loop() centre")
    with open(os.path.join(out, "initial_conditions.cpp"), "w") as f:
        f.write(ic)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
