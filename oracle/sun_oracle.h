/*
 * sun_oracle.h -- FP64 CPU restatement of the CULQCD (nmrcardoso/sun) hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA engine
 * is compared against, and the CPU baseline that bench.py times.  The product
 * (sun_b200/libsun_b200.so) never links, loads or calls it.
 *
 * Host lattice format ("canonical"): double complex U[V][4][N][N], sites in
 * lexicographic order lex = x + X0*(y + X1*(z + X2*t)), each link an N x N
 * row-major complex matrix.  This is exactly the record order of the
 * reference's SaveBin_Gauge file body (io_gauge.cpp:544-563).
 *
 * Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3", SC'11), keyed and countered exactly like the
 * CUDA engine:
 *     key     = (seed & 0xffffffff, seed >> 32)
 *     counter = (block, lex_site, mu | purpose << 8, pass)
 * where `block` increments every 4 words of a link's stream and `pass` is the
 * lattice's heatbath-pass counter (0 for the hot start).  A uniform in FP32
 * mode takes one word w: u = ((w >> 8) + 1) * 2^-24, in (0, 1].  In FP64 mode
 * it takes two words a, b: u = ((((a >> 11) << 32) | b) + 1) * 2^-53.
 */
#ifndef SUN_ORACLE_H
#define SUN_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* uniform-stream modes */
#define ORC_RNG_PHILOX32 0   /* FP32 engine: one Philox word per uniform */
#define ORC_RNG_PHILOX64 1   /* FP64 engine: two Philox words per uniform */
#define ORC_RNG_INJECTED 2   /* uniforms read from a caller buffer          */

/* link layouts of the device image (reference ArrayType, modes.h:66-71) */
#define ORC_SOA   0
#define ORC_SOA12 1
#define ORC_SOA8  2

/* --- random numbers ----------------------------------------------------- */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* n uniforms of the stream of link (lex, mu) for heatbath pass `pass`. */
void orc_uniforms(uint64_t seed, int lex, int mu, int purpose, uint32_t pass,
                  int fp64, int n, double *out);

/* --- SU(N) helpers ---------------------------------------------------------*/
void orc_su2_index(int N, int block, int *p, int *q);
void orc_reunit_link(int N, double *U /* N*N complex, interleaved */);
/* one heatbath / overrelaxation update of one link given F = staple^dagger.
 * For heatbath the uniform stream is (mode, seed, lex, mu, pass) or an
 * injected buffer inj[0..inj_len).  Returns the number of uniforms used, or
 * -1 if the injected buffer ran out. */
int  orc_heatbath_link(int N, double *U, const double *F, double beta_over_n,
                       int mode, uint64_t seed, int lex, int mu, uint32_t pass,
                       const double *inj, int inj_len);
void orc_overrelax_link(int N, double *U, const double *F);
void orc_su2_generate(double alpha, int mode, uint64_t seed, int lex, int mu,
                      uint32_t pass, const double *inj, int inj_len, double a[4], int *used);

/* --- lattice operations (canonical layout) ---------------------------------*/
void orc_cold(int N, const int X[4], double *U);
void orc_hot(int N, const int X[4], double *U, uint64_t seed);
void orc_staple(int N, const int X[4], const double *U, int lex, int mu, double *S);
/* one (parity, mu) phase.  kind 0 = heatbath, 1 = overrelaxation.
 * inj: uniforms per link, inj[(lex*4+mu)*inj_stride + k]. Returns the number
 * of links whose injected stream ran out (0 on success). */
int  orc_update_phase(int N, const int X[4], double *U, int parity, int mu, int kind,
                      double beta, int mode, uint64_t seed, uint32_t pass,
                      const double *inj, int inj_stride, int nthreads);
/* n_sweeps x (n_hb heatbath + n_or overrelaxation) passes; pass counter
 * starts at *pass and is advanced by n_hb per sweep.  reunit_every > 0
 * reunitarizes after every reunit_every-th sweep. */
void orc_sweeps(int N, const int X[4], double *U, double beta, int n_hb, int n_or,
                int n_sweeps, int reunit_every, int mode, uint64_t seed, uint32_t *pass,
                int nthreads);
void orc_reunitarize(int N, const int X[4], double *U);
double orc_unitarity_violation(int N, const int X[4], const double *U);
void orc_link_trace_det(int N, const int X[4], const double *U, double out[4]);

/* --- measurements -----------------------------------------------------------*/
void orc_plaquette(int N, const int X[4], const double *U, double out[2]);
void orc_polyakov(int N, const int X[4], const double *U, double out[2]);
void orc_wilson_loops(int N, const int X[4], const double *U, int R, int T, double *out);

/* --- device-image layout ------------------------------------------------------*/
int  orc_layout_elems(int N, int layout);
/* canonical -> device image (complex elements of `fp64 ? 16 : 8` bytes) */
void orc_pack(int N, const int X[4], const double *U, int layout, int evenodd, int fp64, void *img);
/* device image -> canonical (reconstructing 12/8-parameter links) */
void orc_unpack(int N, const int X[4], const void *img, int layout, int evenodd, int fp64, double *U);

/* --- reference gauge file (SaveBin_Gauge / ReadBin_Gauge) -------------------*/
int  orc_save_bin(int N, const int X[4], const double *U, double beta, const char *path,
                  int save_fp64, int header_fp64, int with_header);
int  orc_load_bin(int N, const int X[4], double *U, const char *path, int save_fp64,
                  int header_fp64, int with_header, int grid_out[4], double *beta_out);

/* --- smearing and multihit (sun_oracle_smear.inc) ---------------------------
 * dirmask: bit mu selects direction mu (7 = space, 8 = time). */
void orc_project_sun(int N, double *W, const double *Q, int nhits, double tol);
void orc_exp_iq3(const double *Q, double *E);
void orc_ape(int N, const int X[4], double *U, double w, int steps, int nhits, double tol, int dirmask);
void orc_stout(const int X[4], double *U, double w, int steps, int dirmask);
void orc_hyp(int N, const int X[4], double *U, const float alpha[3], int steps, int nhits, double tol,
             int dirmask);
void orc_multihit(int N, const int X[4], const double *Uin, double *Uout, double beta, int nhit,
                  int mode, uint64_t seed);
void orc_multihit_space(int N, const int X[4], const double *Uin, double *Uout, int nhit);

#ifdef __cplusplus
}
#endif
#endif
