// fused.h — scratch layouts and launch helpers of the fused DOT and CSRMV,
// shared by their host wrappers and the graph-captured CG.
#pragma once
#include "chain.cuh"
#include "ozb_internal.h"

namespace ozb {

constexpr int kDotLevels = kChainLevels;
constexpr int kDotThreads = 256;
constexpr int kDotStages = 8;  // cp.async stages per thread (dynamic shared memory)

struct alignas(8) DotStatus {  // copied to the host in one piece
    int status, ns0, ns1, pad;
    double result;
};

constexpr int kDotDigitRows = 32;  // levels x digits per vector in the tensor-core pass (at most)

struct DotScratch {
    VecStats vs;                        // first pass: max, lowest set bit, Inf/NaN of x and y
    double P[kDotLevels * kDotLevels];  // exact slice products P[ia * 8 + ib]
    long long T[kDotDigitRows * kDotDigitRows];  // tensor-core pass: digit-pair sums T[p * 32 + q]
    unsigned proven[2];                 // levels whose predicted tau some element proved
    unsigned ticket;                    // blocks of pass 2 that are done
    int err;                            // tensor-core pass: a bounded wait ran out
    DotStatus out;
};

constexpr int kCsrLv = kChainLevels;  // levels of x computed / proven
constexpr int kCsrRowMax = 8;         // entries per row held on chip
constexpr int kCsrThreads = 128;

struct CsrScratch {
    VecStats vs;                 // first pass over x
    unsigned proven;             // levels of x's chain whose predicted tau some element proved
    unsigned ticket;             // blocks of the proof pass that are done
    int valid, nB, nslow, zmax;  // zmax: first zero-remainder level of A, max over rows
    int xcomplete;               // x's (proven) split is complete: its last remainder is zero
    int rn_declined;             // the correctly rounded row kernel wrote nothing (x's split incomplete)
    double sigma[kCsrLv];        // x's proven sigmas
};

// DOT: the first pass (max, lowest set bit) into sc->vs, and the second
// pass, which leaves the result and status in sc->out and its accumulators
// zeroed.  `gate` (device int, may be null): the kernel does nothing when 0.
int dot_scan_launch(cudaStream_t s, int nsm, int n, const double *x, const double *y, DotScratch *sc);
int dot_tree_launch(cudaStream_t s, int nsm, int n, const double *x, const double *y, int rho, int maxS,
                    int sum_mode, DotScratch *sc, const int *gate,
                    bool tree_only = false);
// Sets the kernels' shared-memory attribute up front (before a capture).
int dot_tree_prepare();
// The tensor-core form of pass 2 (dot_i8.cu): digits per level for rho (0:
// not applicable), its launch (every valid plan) and its shared-memory
// attributes.
int dot_i8_digits(int rho);
int dot_i8_launch(cudaStream_t s, int nsm, int n, const double *x, const double *y, int rho, int maxS,
                  int sum_mode, DotScratch *sc, const int *gate);
int dot_i8_prepare();


// CSRMV pieces (csrmv_fused.cu): statistics of a vector into vs[index]; the
// rows the row kernel defers (a property of the matrix); proof of x's chain
// (publishes sc->valid, nB, sigma, zeroes sc->vs); the row kernel.  With
// `fixed_slow` >= 0 the deferred rows are the given list (no appends);
// `ystats` (may be null) collects max / lowest bit of the written y.
struct CsrmvArgs {
    int m, n;
    double alpha, beta;
    const double *val;
    const int *colind, *rowptr;
    const double *x;
    double *y;
    int shift, epsmode, maxS, sum_mode, na_hint;
};
int vec_stats_launch(cudaStream_t s, int nsm, int n, const double *x, VecStats *vs, int index);
int csr_slow_rows_launch(cudaStream_t s, int m, const double *val, const int *rowptr, int shift, int epsmode,
                         int maxS, int na_hint, int *list, int *count);
int csr_proof_launch(cudaStream_t s, int n, const double *x, int rho, int maxS, CsrScratch *sc, const int *gate);
int csr_rows_launch(cudaStream_t s, const CsrmvArgs &a, CsrScratch *sc, int *slow, int fixed_slow,
                    VecStats *ystats, int ystats_index, double *terms, const int *gate);
// NearSum rows as the correctly rounded exact row dots (csrmv_fused.cu): true
// when the arguments allow it (sum mode 1, splitEpsMode 0, a power-of-two
// shift).  The kernel writes nothing when x's split is incomplete
// (sc->rn_declined); rows whose split is incomplete or whose slice products
// could be inexact are appended to the slow list, or with a fixed list
// (fixed_slow >= 0, whose rows the call computes afterwards) they decline the
// whole product (sc->rn_declined).
bool csr_rn_applies(const CsrmvArgs &a);
// With `xstats` (x's statistics at index 0) the kernel decides x's completeness
// itself and needs no proof (no fixed list then: its rows need x's proven chain).
int csr_rn_launch(cudaStream_t s, const CsrmvArgs &a, CsrScratch *sc, int *slow, int fixed_slow, VecStats *ystats,
                  int ystats_index, double *terms, const int *gate, const VecStats *xstats = nullptr);

}  // namespace ozb
