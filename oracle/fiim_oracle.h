/* ORACLE TEST INFRASTRUCTURE — not product code.
 *
 * Plain-C, single-threaded restatement of the reference's BiCGSTAB solve phase
 * with the factored approximate inverse z = G * D^{-1} * (H * r). Only tests/,
 * smoke() and bench.py's CPU-baseline leg may load it, and only as the checker.
 * Every routine cites the reference lines it restates; see fiim_oracle.c.
 *
 * Pinned against the reference itself: tests/test_oracle.py runs the reference's
 * own EPBiCGSTAB / PBiCGSTAB (compiled unmodified against oracle/mkl_shim, one
 * thread) beside these routines and requires bit-identical x, iteration count,
 * info and residual. MKL's own arithmetic stays unpinned: MKL is absent here and
 * no reference test fixes its results (the reference has no tests).
 */
#ifndef FIIM_ORACLE_H
#define FIIM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Package whose EPBiCGSTAB/PBiCGSTAB control flow is restated. */
enum { ORC_AFIIM = 0, ORC_PDFIIM = 1, ORC_ACIFIM = 2 };

/* Fill-mode filters, as MKL TRIANGULAR descriptors apply them. */
enum { ORC_GENERAL = 0, ORC_UPPER = 1, ORC_LOWER = 2 };

void orc_csr_mv(int n, const int *Ai, const int *Aj, const double *Av, int fill,
                const double *x, double *y);
void orc_csr_mv_trans(int n, const int *Ai, const int *Aj, const double *Av, int fill,
                      const double *x, double *y);
void orc_csr_mv_sym_upper(int n, const int *Ai, const int *Aj, const double *Av,
                          const double *x, double *y);

void orc_prec_apply(int n, const int *Gi, const int *Gj, const double *Gv, const double *IDv,
                    const int *Hi, const int *Hj, const double *Hv, const double *in,
                    double *out, double *tm);
void orc_prec_apply_sym(int n, const int *Gi, const int *Gj, const double *Gv,
                        const double *IDv, const double *in, double *out, double *tm);
void orc_prec_apply_combined(int n, int nr, const int *Gi, const int *Gj, const double *Gv,
                             const double *IDv, const int *Hi, const int *Hj, const double *Hv,
                             const int *Li, const int *Lj, const double *Lv, const int *Ui,
                             const int *Uj, const double *Uv, const double *in, double *out,
                             double *work);

/* Split every dot product and norm into `blocks` contiguous blocks (see fiim_oracle.c);
 * 1 restores the left-to-right sum. */
void orc_set_dot_blocks(int blocks);

/* One full solve. variant: ORC_*; issym (PDFIIM only): A holds its upper triangle and
 * G^T replaces H; mode (ACIFIM only): 'E' explicit or 'C' combined with nr steps.
 * Returns 0, or -1 on an unsupported argument. */
int orc_bicgstab(int variant, int issym, char mode, int nr, int n, const int *Ai, const int *Aj,
                 const double *Av, const double *b, double tol, int NMAX, const int *Gi,
                 const int *Gj, const double *Gv, const double *IDv, const int *Hi,
                 const int *Hj, const double *Hv, const int *Li, const int *Lj,
                 const double *Lv, const int *Ui, const int *Uj, const double *Uv, double *x,
                 double *resval, int *iter, int *info);

#ifdef __cplusplus
}
#endif
#endif
