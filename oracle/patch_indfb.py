"""Patched copies of reference sources for the applied induction fallback.

The reference's induction corrector (src/induction_ader.hpp:533-563, the
FV_Update_solution method) forms the sub-cell FV update of the face
averages, fills the FV ghosts and detects troubles, but applies no fallback
for B (its fallback_fluxes() call is commented out). The CUDA solver's
optional applied fallback (spdk_induction_config.fallback_apply) replaces,
on every sub-cell edge that touches a troubled cell, the high-order edge
EMF by the first-order upwind EMF of the slice-start face averages, and
redoes the face update from the slice-start faces. This recipe writes
copies of induction_ader.hpp (with that step added after the detection),
spd_k.hpp and main.cpp (unchanged, copied only so that their quoted
includes resolve to the patched header) into the build folder
(oracle/_ref/indfb/, git-ignored); they are compiled with the other
reference objects into oracle/_ref/spd_K_indfb (oracle/Makefile, target
indfb), whose runs with job/fallback=true pin the applied fallback.
Test infrastructure only.

The added step, in the reference's own arrays: for an edge of direction d
(E = Ex, Ey or Ez), d1 = the next direction and d2 the one after, b1 the
FV face array normal to d1 and b2 the one normal to d2 (By_old/Bz_old for
Ex, ...), an edge (k, j, i) touches the four cells (k, j, i) minus 0 or 1
steps along d1 and along d2; if the aggregate trouble slot of any is
non-zero, E(k, j, i) = v1 upwind(b2[-d1], b2, v1) - v2 upwind(b1[-d2], b1, v2)
with v = (1, 1, 0) (src/induction.cpp:29-31) and the reference's upwind()
rule (src/induction.cpp:503-506). The edges covered are those the face
update of the active cells reads: an index in [2, Nx-3] along d
(cell-centred there), [2, Nx-2] across it (Nx = the FV cell count with 2
ghost layers). The patched code names its indices kc, jc, ic because the
reference defines K, J and I as macros.

    python oracle/patch_indfb.py <reference src dir> <output dir>
"""
import os
import sys


def patch(text, old, new, what):
    if text.count(old) != 1:
        raise SystemExit(f"patch_indfb: the {what} text was not found exactly once")
    return text.replace(old, new)


ADDED_METHODS = r"""
    // applied induction fallback (written by oracle/patch_indfb.py)
    std::vector<double> spdk_faces[3];
    void spdk_save_faces(){
        SD_Solution* f[3] = {&Bx, &By, &Bz};
        for(int d=0; d<3; d++)
            spdk_faces[d].assign(f[d]->Vector.data(), f[d]->Vector.data() + f[d]->Vector.size());
    }
    static double spdk_upwind(double l, double r, double v){
        if(v==0) return 0.5*(l+r);
        return v > 0 ? l : r;
    }
    void spdk_fallback_emf(FV_Solution E, FV_Solution B1, FV_Solution B2, int dim){
        const int fx = troubles.Nx, fy = troubles.Ny, fz = troubles.Nz;
        const int Mx = (dim==0 ? fx-3 : fx-2) - 1;
        const int My = (dim==1 ? fy-3 : fy-2) - 1;
        const int Mz = (dim==2 ? fz-3 : fz-2) - 1;
        const int agg = troubles.n_var-1;
        const int d1 = (dim+1)%3, d2 = (dim+2)%3;
        const int o1[3] = {d1==0, d1==1, d1==2}, o2[3] = {d2==0, d2==1, d2==2};
        const double v1 = d1<2 ? 1.0 : 0.0, v2 = d2<2 ? 1.0 : 0.0;
        for(int kc=2; kc<2+Mz; kc++)
        for(int jc=2; jc<2+My; jc++)
        for(int ic=2; ic<2+Mx; ic++){
            double tr = 0;
            for(int s1=0; s1<2; s1++)
            for(int s2=0; s2<2; s2++){
                const double t = troubles.Vector(agg, kc-s1*o1[2]-s2*o2[2], jc-s1*o1[1]-s2*o2[1], ic-s1*o1[0]-s2*o2[0]);
                if(t > tr) tr = t;
            }
            if(tr > 0){
                const double b2L = B2.Vector(0, kc-o1[2], jc-o1[1], ic-o1[0]), b2R = B2.Vector(0, kc, jc, ic);
                const double b1L = B1.Vector(0, kc-o2[2], jc-o2[1], ic-o2[0]), b1R = B1.Vector(0, kc, jc, ic);
                E.Vector(0, kc, jc, ic) = v1*spdk_upwind(b2L, b2R, v1) - v2*spdk_upwind(b1L, b1R, v2);
            }
        }
    }
    void spdk_apply_fallback(int ader, dimension X_dim, dimension Y_dim, dimension Z_dim){
        spdk_fallback_emf(Ex, By_old, Bz_old, 0);
        spdk_fallback_emf(Ey, Bz_old, Bx_old, 1);
        spdk_fallback_emf(Ez, Bx_old, By_old, 2);
        SD_Solution* f[3] = {&Bx, &By, &Bz};
        for(int d=0; d<3; d++)
            std::copy(spdk_faces[d].begin(), spdk_faces[d].end(), f[d]->Vector.data());
        FV_update_solution(ader, X_dim.fv_faces, Y_dim.fv_faces, Z_dim.fv_faces, 1);
    }

"""


def main(src, out):
    os.makedirs(out, exist_ok=True)
    with open(os.path.join(src, "induction_ader.hpp")) as f:
        h = f.read()
    h = patch(h, "            Integrate_edges(ader);\n            FV_update_solution(ader, X_dim.fv_faces, "
                 "Y_dim.fv_faces, Z_dim.fv_faces, 1);\n",
              "            Integrate_edges(ader);\n            spdk_save_faces();\n"
              "            FV_update_solution(ader, X_dim.fv_faces, Y_dim.fv_faces, Z_dim.fv_faces, 1);\n",
              "corrector face update")
    h = patch(h, "        //    //fallback_fluxes();\n",
              "            spdk_apply_fallback(ader, X_dim, Y_dim, Z_dim);\n        //    //fallback_fluxes();\n",
              "commented-out fallback")
    h = patch(h, "    void FV_update_solution(int ader, Vector xs, Vector ys, Vector zs, bool update){\n",
              ADDED_METHODS + "    void FV_update_solution(int ader, Vector xs, Vector ys, Vector zs, bool update){\n",
              "FV_update_solution")
    with open(os.path.join(out, "induction_ader.hpp"), "w") as f:
        f.write(h)
    for name in ("spd_k.hpp", "main.cpp"):
        with open(os.path.join(src, name)) as f:
            t = f.read()
        with open(os.path.join(out, name), "w") as f:
            f.write(t)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
