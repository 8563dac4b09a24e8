"""Build the reference SWEHR program into oracle/_ref/ (TEST INFRASTRUCTURE).

Reads SWEHR.c from the reference checkout named by --reference or by the
environment variable SWEHR_REFERENCE (no default: a missing checkout is an
error), applies the small set of patches below, writes the patched
copy to oracle/_ref/swehr_ref.c and compiles two binaries:

  oracle/_ref/swehr_ref      serial, exactly the reference's arithmetic
  oracle/_ref/swehr_ref_omp  the reference's own (commented-out) OpenMP
                             pragmas switched on, with the max-reduction of
                             Smax/velmax they lack (SWEHR.c:1091,1416); this
                             is the timed CPU baseline

Patches (every one is a no-op with the default swehr_ref.cfg, except
zero-initialised allocation, which is what fresh heap pages give the stock
program anyway):
  1. NR allocators use calloc (SWEHR.c:38-198) -- the reference reads U[1],
     M, TOTM, DEP, TOTSED, SOLID before writing them.
  2. BNDRY, the j=ny inflow switch, per-cell soil constants (roughness, Ks
     (optionally per cell from ks.txt), theta0, thetas, hf, initial VINF,
     UC, UC2), a step limit and a movie switch are read from swehr_ref.cfg
     in the working directory when it exists (SWEHR.c:236-246, 617-621,
     1010-1035, 808, 1679).
  3. Sample points and the second outlet row are clamped to the grid
     (SWEHR.c:699, 710-715 read out of bounds when ny < 50).
  4. After the loop: elapsed time via omp_get_wtime, step count, and a
     %.17g dump of every state field to swehr_dump.txt.
  5. The deposit cohesion (SWEHR.c:647) and an interior SOLID mask
     (solid.txt, nx*ny integers i-major; the stock program leaves SOLID all
     zero, SWEHR.c:597) come from swehr_ref.cfg as well, so slope failure
     and interior walls can be exercised.  Every int matrix gets one spare
     zero row: the y-face solid test reads SOLID[nx][ny+1], one element past
     the stock allocation (SWEHR.c:1206,1211).

Run:  SWEHR_REFERENCE=<checkout> python oracle/build_ref.py   (or --reference DIR)
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

HELPERS = r'''
/* ---- build_ref.py: run-time configuration (swehr_ref.cfg) ---- */
static int swehr_cfg_loaded = 0;
static int swehr_cfg_bndry[5] = {0, 1, 0, 1, 1};
static int swehr_cfg_inflow = 1;
static long swehr_cfg_maxsteps = -1;
static int swehr_cfg_movies = 1;
static int swehr_cfg_dump = 1;
static double swehr_cfg_roughness = 0.1, swehr_cfg_ks = 0, swehr_cfg_theta0 = 0.05;
static double swehr_cfg_thetas = 0.4, swehr_cfg_hf = 0.001, swehr_cfg_vinf0 = 1e-4;
static double swehr_cfg_uc = 0, swehr_cfg_uc2 = 0;
static int swehr_cfg_ksfile = 0;
static double *swehr_cfg_ksvals = 0;
static int swehr_cfg_set_cohesion = 0;
static double swehr_cfg_cohesion = 400;
static int swehr_cfg_solidfile = 0;
static int *swehr_cfg_solidvals = 0;
static long swehr_steps = 0;
static void swehr_cfg_load(void)
{
    FILE *f;
    char key[64];
    double v;
    if (swehr_cfg_loaded) return;
    swehr_cfg_loaded = 1;
    f = fopen("./swehr_ref.cfg", "r");
    if (!f) return;
    while (fscanf(f, "%63s %lf", key, &v) == 2) {
        if (!strcmp(key, "bndry1")) swehr_cfg_bndry[1] = (int)v;
        else if (!strcmp(key, "bndry2")) swehr_cfg_bndry[2] = (int)v;
        else if (!strcmp(key, "bndry3")) swehr_cfg_bndry[3] = (int)v;
        else if (!strcmp(key, "bndry4")) swehr_cfg_bndry[4] = (int)v;
        else if (!strcmp(key, "inflow")) swehr_cfg_inflow = (int)v;
        else if (!strcmp(key, "maxsteps")) swehr_cfg_maxsteps = (long)v;
        else if (!strcmp(key, "movies")) swehr_cfg_movies = (int)v;
        else if (!strcmp(key, "dump")) swehr_cfg_dump = (int)v;
        else if (!strcmp(key, "roughness")) swehr_cfg_roughness = v;
        else if (!strcmp(key, "ks")) swehr_cfg_ks = v;
        else if (!strcmp(key, "ksfile")) swehr_cfg_ksfile = (int)v;
        else if (!strcmp(key, "theta0")) swehr_cfg_theta0 = v;
        else if (!strcmp(key, "thetas")) swehr_cfg_thetas = v;
        else if (!strcmp(key, "hf")) swehr_cfg_hf = v;
        else if (!strcmp(key, "vinf0")) swehr_cfg_vinf0 = v;
        else if (!strcmp(key, "uc")) swehr_cfg_uc = v;
        else if (!strcmp(key, "uc2")) swehr_cfg_uc2 = v;
        else if (!strcmp(key, "cohesion")) { swehr_cfg_cohesion = v; swehr_cfg_set_cohesion = 1; }
        else if (!strcmp(key, "solidfile")) swehr_cfg_solidfile = (int)v;
    }
    fclose(f);
}
static double swehr_cfg_ks_at(int i, int j, int nx, int ny)
{
    swehr_cfg_load();
    if (!swehr_cfg_ksfile) return swehr_cfg_ks;
    if (!swehr_cfg_ksvals) {
        FILE *f = fopen("./ks.txt", "r");
        long n, q;
        n = (long)nx * ny;
        swehr_cfg_ksvals = (double *)calloc(n, sizeof(double));
        for (q = 0; q < n; q++)
            if (fscanf(f, "%lf", &swehr_cfg_ksvals[q]) != 1) break;
        fclose(f);
    }
    return swehr_cfg_ksvals[(long)(i - 1) * ny + (j - 1)];
}
static int swehr_cfg_solid_at(int i, int j, int nx, int ny)
{
    swehr_cfg_load();
    if (!swehr_cfg_solidfile) return 0;
    if (!swehr_cfg_solidvals) {
        FILE *f = fopen("./solid.txt", "r");
        long n, q;
        n = (long)nx * ny;
        swehr_cfg_solidvals = (int *)calloc(n, sizeof(int));
        for (q = 0; q < n; q++)
            if (fscanf(f, "%d", &swehr_cfg_solidvals[q]) != 1) break;
        fclose(f);
    }
    return swehr_cfg_solidvals[(long)(i - 1) * ny + (j - 1)];
}
'''

DUMP = r'''
    {
        double swehr_el = omp_get_wtime() - swehr_w0;
        printf("SWEHR_REF steps %ld elapsed %.6f threads %d t %.17g\n", swehr_steps, swehr_el, omp_get_max_threads(), t);
        if (swehr_cfg_dump) {
            FILE *fd = fopen("./swehr_dump.txt", "w");
            int ii, jj, kk;
            fprintf(fd, "%d %d %d %ld %.17g\n", nx, ny, sclass, swehr_steps, t);
#define SWEHR_DUMP2(A) for (ii=1;ii<=nx;ii++) for (jj=1;jj<=ny;jj++) fprintf(fd, "%.17g\n", (A)[ii][jj]);
            SWEHR_DUMP2(U[1]) SWEHR_DUMP2(U[2]) SWEHR_DUMP2(U[3]) SWEHR_DUMP2(TOPO) SWEHR_DUMP2(VINF)
            SWEHR_DUMP2(TOTM) SWEHR_DUMP2(DEP) SWEHR_DUMP2(TOTSED) SWEHR_DUMP2(MAXVEL) SWEHR_DUMP2(MAXDEPTH)
            for (kk=4;kk<=nn;kk++) { SWEHR_DUMP2(U[kk]) }
            for (kk=1;kk<=sclass;kk++) { SWEHR_DUMP2(M[kk]) }
            for (kk=1;kk<=sclass;kk++) { SWEHR_DUMP2(SED[kk]) }
            fprintf(fd, "%d\n", stagecnt);
            for (jj=1;jj<=stagecnt;jj++) for (ii=1;ii<=24;ii++) fprintf(fd, "%.17g\n", STAGE[ii][jj]);
            for (jj=1;jj<=stagecnt;jj++) for (ii=1;ii<=18;ii++) fprintf(fd, "%.17g\n", SAVEFLOW[ii][jj]);
            fclose(fd);
        }
    }
'''

# (anchor, replacement, expected count)
PATCHES = [
    ("#include<stdlib.h>\n", "#include<stdlib.h>\n#include<string.h>\n", 1),
    ("malloc(", "calloc(1,", None),
    # one spare row of zeros behind every int matrix: the y-face solid test
    # reads SOLID[i][ny+1] (SWEHR.c:1206,1211), one int past the allocation at i = nx
    ("(nrow*ncol+NR_END)*sizeof(int)", "(nrow*ncol+NR_END+ncol)*sizeof(int)", 1),
    ("            fscanf(fr0,\"%lf\",&TOPO[i][j]);      // TOPOGRAPHY\n",
     "            fscanf(fr0,\"%lf\",&TOPO[i][j]);      // TOPOGRAPHY\n"
     "            SOLID[i][j]=swehr_cfg_solid_at(i,j,nx,ny);\n", 1),
    ("    cohesion=400;", "    cohesion=400; swehr_cfg_load(); if (swehr_cfg_set_cohesion) cohesion=swehr_cfg_cohesion;", 1),
    ("void initialcondition(", HELPERS + "\nvoid initialcondition(", 1),
    ("            MANNING[i][j]=0.1;", "            swehr_cfg_load();\n            MANNING[i][j]=swehr_cfg_roughness;", 1),
    ("            ROUGHNESS[i][j]=0.1;", "            ROUGHNESS[i][j]=swehr_cfg_roughness;", 1),
    ("            KS[i][j]=0;", "            KS[i][j]=swehr_cfg_ks_at(i,j,nx,ny);", 1),
    ("            THETA0[i][j]=0.05;", "            THETA0[i][j]=swehr_cfg_theta0;", 1),
    ("            THETAS[i][j]=0.4;", "            THETAS[i][j]=swehr_cfg_thetas;", 1),
    ("            HF[i][j]=0.001;", "            HF[i][j]=swehr_cfg_hf;", 1),
    ("            VINF[i][j]=1e-4;", "            VINF[i][j]=swehr_cfg_vinf0;", 1),
    ("            UC[i][j]=0;", "            UC[i][j]=swehr_cfg_uc;", 1),
    ("            UC2[i][j]=0;", "            UC2[i][j]=swehr_cfg_uc2;", 1),
    ("    BNDRY[4]=1;                                 // B.C. at j==ny\n",
     "    BNDRY[4]=1;                                 // B.C. at j==ny\n"
     "    swehr_cfg_load();\n    for (k=1;k<=4;k++) BNDRY[k]=swehr_cfg_bndry[k];\n", 1),
    ("    outlet2=1; outlety2=10;", "    outlet2=1; outlety2=(10<ny?10:ny);", 1),
    ("    for (k=1;k<=6;k++)\n        printf(",
     "    for (k=1;k<=6;k++) { if (XPOINT[k]>nx) XPOINT[k]=nx; if (YPOINT[k]>ny) YPOINT[k]=ny; }\n"
     "    for (k=1;k<=6;k++)\n        printf(", 1),
    ("    time_t t0 = time(NULL);\n", "    time_t t0 = time(NULL);\n    double swehr_w0 = omp_get_wtime();\n", 1),
    ("    while (t<tend)\n", "    while (t<tend && (swehr_cfg_maxsteps < 0 || swehr_steps < swehr_cfg_maxsteps))\n", 1),
    ("        // Sediment and Water Inflow B.C. at j=ny\n        for (i=-1;i<=nx+2;i++)",
     "        // Sediment and Water Inflow B.C. at j=ny\n        if (swehr_cfg_inflow) for (i=-1;i<=nx+2;i++)", 1),
    ("        //#pragma omp parallel for private(j,k,Smaxtemp,ULR,TFLUX,q,beta,mtstar,pgfx,pgfy)\n",
     "#ifdef SWEHR_REF_OMP\n#pragma omp parallel for private(j,k,Smaxtemp,ULR,TFLUX,q,beta,mtstar,pgfx,pgfy) reduction(max:Smax,velmax)\n#endif\n", 1),
    ("        //#pragma omp parallel for private(j,k,chtemp,redetach,beta)\n",
     "#ifdef SWEHR_REF_OMP\n#pragma omp parallel for private(j,k,chtemp,redetach,beta)\n#endif\n", 1),
    ("        t+=dt;\n", "        t+=dt;\n        swehr_steps++;\n", 1),
    ("        if (t>stageinterval)\n", "        if (t>stageinterval && stagecnt < 29999)\n", 1),
    ("        if (t>=printinterval)\n", "        if (swehr_cfg_movies && t>=printinterval)\n", 1),
    ("    time_t t1 = time(NULL);\n", "    time_t t1 = time(NULL);\n" + DUMP, 1),
]


def patch(src: str) -> str:
    for anchor, repl, count in PATCHES:
        n = src.count(anchor)
        if count is not None and n != count:
            raise SystemExit(f"build_ref: anchor found {n}x (want {count}): {anchor[:60]!r}")
        if n == 0:
            raise SystemExit(f"build_ref: anchor missing: {anchor[:60]!r}")
        src = src.replace(anchor, repl)
    return src


def build(reference: str, quiet: bool = False) -> bool:
    src_path = os.path.join(reference, "SWEHR.c")
    if not os.path.exists(src_path):
        if not quiet:
            print(f"build_ref: {src_path} not found; skipping", file=sys.stderr)
        return False
    os.makedirs(OUT, exist_ok=True)
    with open(src_path) as f:
        src = f.read()
    out_c = os.path.join(OUT, "swehr_ref.c")
    with open(out_c, "w") as f:
        f.write(patch(src))
    cmds = [
        ["gcc", "-O2", "-fopenmp", "-w", "-o", os.path.join(OUT, "swehr_ref"), out_c, "-lm"],
        ["gcc", "-O2", "-fopenmp", "-w", "-DSWEHR_REF_OMP", "-o", os.path.join(OUT, "swehr_ref_omp"), out_c, "-lm"],
    ]
    for cmd in cmds:
        subprocess.check_call(cmd)
    if not quiet:
        print("build_ref: built", ", ".join(c[c.index("-o") + 1] for c in cmds))
    return True


REFERENCE_ENV = "SWEHR_REFERENCE"


def reference_dir(explicit: str = None) -> str:
    """The reference checkout: `explicit`, else $SWEHR_REFERENCE; raises
    with a clear message when neither names a directory holding SWEHR.c."""
    d = explicit or os.environ.get(REFERENCE_ENV)
    if not d:
        raise SystemExit(f"build_ref: no reference checkout given: pass --reference DIR or set {REFERENCE_ENV}")
    if not os.path.exists(os.path.join(d, "SWEHR.c")):
        raise SystemExit(f"build_ref: {d} holds no SWEHR.c")
    return d


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help=f"reference checkout (default: ${REFERENCE_ENV})")
    a = ap.parse_args()
    ok = build(reference_dir(a.reference))
    sys.exit(0 if ok else 1)


if __name__ == "__main__":
    main()
