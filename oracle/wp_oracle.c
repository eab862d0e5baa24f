/*
 * wp_oracle.c -- FP64 CPU oracle of the WaveletPotentials projection-and-recovery path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg.  Nothing in the product library calls it.
 *
 * Each routine cites the reference file:line it restates (paths relative to the reference
 * project's WaveletPotentials/ directory).  The lifting constants and base-level matrices are
 * tables that must be identical to the reference's (cuWaveletCompute.cuh); they are written
 * out here as data.
 */
#include "wp_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* OpenMP threads of the parallel loops (the oracle's results do not depend on the count beyond
   the order of the norm reductions) */
void or_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
int or_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

#define HALO 6
#define EPS12 1e-12

/* ---------------------------------------------------------------- lifting constants ---- */
/* CDF3.7 ("curl" wavelet): cuWaveletCompute.cuh:13-23 (Q5 predict/update, Q7 long update) */
static const double Q5_FU1 = -1.0 / 3.0;
static const double Q5_FP[2] = {-3.0 / 8.0, -9.0 / 8.0};
static const double Q7_FU2[7] = {-0.003797743055556, 0.032552083333333, -0.137044270833333, 0.444444444444444,
                                 0.137044270833333, -0.032552083333333, 0.003797743055556};
static const double Q5_SCL[2] = {3.0 / 1.414213562373095048801, 1.414213562373095048801 / 3.0};
/* CDF4.6 ("div" wavelet): cuWaveletCompute.cuh:139-148 */
static const double C4_FU1[2] = {-0.25, -0.25};
static const double C4_FP[2] = {-1.0, -1.0};
static const double C6_FU2[6] = {0.008544921875000, -0.064697265625000, 0.243652343750000,
                                 0.243652343750000, -0.064697265625000, 0.008544921875000};
#define SQ2 1.41421356237309504880168872420969807856967187537694
static const double C4_SCL[2] = {2.0 * SQ2, -1.0 / (2.0 * SQ2)};
static const double C4_SCL_INV[2] = {1.0 / (2.0 * SQ2), -(2.0 * SQ2)};
/* CDF4.4: CDF4.6's first update, predict and scaling with a 4-tap second update
   (cuWaveletCompute.cuh:139-148, cuUpdateCdf44_ad :376-390, cuUpdateCdf44_ad_i :753-769) */
static const double C4_FU2[4] = {-0.03906250, 0.22656250, 0.22656250, -0.03906250};
/* CDF2.6 / CDF2.8: one predict and one update (cuWaveletCompute.cuh:72-81; cuUpdateCdf26_ad :313-334,
   cuUpdateCdf26_ad_i :700-717, cuUpdateCdf28_ad :902-924, cuUpdateCdf28_ad_i :966-984) */
static const double L6_FP[2] = {-0.5, -0.5};
static const double L6_FU[6] = {0.009765625, -0.076171875, 0.31640625, 0.31640625, -0.076171875, 0.009765625};
static const double L8_FU[8] = {-0.002136230468750, 0.020446777343750, -0.095397949218750, 0.327087402343750,
                                0.327087402343750, -0.095397949218750, 0.020446777343750, -0.002136230468750};
static const double L6_SCL[2] = {SQ2, 1.0 / SQ2};

/* base-level matrices, row-major: cuWaveletCompute.cuh:773-797 (CDF3.7), :846-874 (CDF4.6) */
/* CDF3.5 (cuWaveletCompute.cuh:15 RSW_Q5_fu_2, :34-45 RSW_QN5_L10 / RSW_iQN5_L10, :60-71 RSW_QD5_L10 /
   RSW_iQD5_L10); the first update, predict and scaling are CDF3.7's */
static const double Q5_FU2[5] = {5. / 288, -34. / 288, 128. / 288, 34. / 288, -5. / 288};
static const double QN5_L10[16] = {0.5, 0.5, 0.5, 0.5, -0.3828125, -0.234375, 0.234375, 0.3828125,
                                   -0.353553390593274, 0.530330085889911, -0.176776695296637, 0,
                                   0, 0.176776695296637, -0.530330085889911, 0.353553390593274};
static const double IQN5_L10[16] = {0.5, -1.0, -1.038563084867742, 0.375650477505353,
                                    0.5, -0.5, 1.248485410532498, -0.165728151840597,
                                    0.5, 0.5, 0.165728151840597, -1.248485410532498,
                                    0.5, 1.0, -0.375650477505353, 1.038563084867742};
static const double QD5_L10[16] = {0.937499999999999, 1.53125, 1.53125, 0.9375, -1.0, -1.0, 1.0, 1.0,
                                   -0.707106781186548, 0.530330085889911, -0.176776695296637, 0,
                                   0, 0.176776695296637, -0.530330085889911, 0.707106781186548};
static const double IQD5_L10[16] = {0.125, -0.25, -0.894932019939224, 0.187825238752677,
                                    0.25, -0.25, 0.685009694274468, 0.02209708691208,
                                    0.25, 0.25, -0.02209708691208, -0.685009694274468,
                                    0.125, 0.25, -0.187825238752677, 0.894932019939224};
#define IS_Q3(w) ((w) == OR_CDF3_7 || (w) == OR_CDF3_5)
static const double QN7_L10[16] = {
    0.500000000000000, 0.500000000000000, 0.500000000000000, 0.500000000000000,
    -0.399902343750000, -0.200195312500000, 0.200195312500000, 0.399902343750000,
    -0.353553390593274, 0.530330085889911, -0.176776695296637, 0,
    0, 0.176776695296637, -0.530330085889911, 0.353553390593274};
static const double IQN7_L10[16] = {
    0.500000000000000, -1.000000000000000, -0.990225707247567, 0.423987855125528,
    0.500000000000000, -0.500000000000000, 1.272654099342585, -0.141559463030510,
    0.500000000000000, 0.500000000000000, 0.141559463030510, -1.272654099342585,
    0.500000000000000, 1.000000000000000, -0.423987855125528, 0.990225707247567};
static const double QD7_L10[16] = {
    0.800781250000000, 1.599609375000000, 1.599609375000000, 0.800781250000000,
    -1.000000000000000, -1.000000000000000, 1.000000000000000, 1.000000000000000,
    -0.707106781186548, 0.530330085889911, -0.176776695296637, 0,
    0, 0.176776695296637, -0.530330085889911, 0.707106781186548};
static const double IQD7_L10[16] = {
    0.125000000000000, -0.250000000000000, -0.919100708749311, 0.211993927562764,
    0.250000000000000, -0.250000000000000, 0.636672316654294, 0.070434464532254,
    0.250000000000000, 0.250000000000000, -0.070434464532254, -0.636672316654294,
    0.125000000000000, 0.250000000000000, -0.211993927562764, 0.919100708749311};
static const double CN6_L10[25] = {
    1.851562500000001, 2.097656250000000, 0.500000000000000, -1.097656250000000, -1.351562500000000,
    -1.351562500000000, -1.097656250000000, 0.500000000000000, 2.097656250000000, 1.851562500000001,
    1.000000000000000, 0.000000000000000, -2.000000000000000, 0.000000000000000, 1.000000000000000,
    0.353553390593274, -0.618718433538229, 0.353553390593274, -0.088388347648318, 0,
    0, -0.088388347648318, 0.353553390593274, -0.618718433538229, 0.353553390593274};
static const double ICN6_L10[25] = {
    0.343750000000000, 0.156250000000000, 0.250000000000000, 0.918410174783309, -0.211303393596761,
    0.312500000000000, 0.187500000000000, 0, -0.919791242715314, 0.212684461528766,
    0.250000000000000, 0.250000000000000, -0.250000000000000, 0.353553390593274, 0.353553390593274,
    0.187500000000000, 0.312500000000000, 0, 0.212684461528766, -0.919791242715314,
    0.156250000000000, 0.343750000000000, 0.250000000000000, -0.211303393596761, 0.918410174783309};
static const double CD6_L10[25] = {
    2.102851867675782, -0.000000000000000, -0.000000000000000, -0.000000000000000, 0.000000000000000,
    -0.000000000000000, 0.000000000000000, 0.000000000000000, 0.000000000000000, 2.102851867675782,
    0.683105468750000, -0.199707031250000, -0.400390625000000, -0.199707031250000, 0.683105468750000,
    0.353553390593274, -0.441941738241592, 0.353553390593274, -0.088388347648318, 0,
    0, -0.088388347648318, 0.353553390593274, -0.441941738241592, 0.353553390593274};
static const double ICD6_L10[25] = {
    0.281250000000000, 0, 0.000000000000000, 0.000000000000000, -0.000000000000000,
    0.312500000000000, 0.125000000000000, -1.000000000000000, -1.980451414495135, 0.847975710251055,
    0.234375000000000, 0.234375000000000, -1.500000000000000, 0.564856784190035, 0.564856784190035,
    0.125000000000000, 0.312500000000000, -1.000000000000000, 0.847975710251055, -1.980451414495135,
    0, 0.281250000000000, -0.000000000000000, 0.000000000000000, -0.000000000000000};

/* base-level matrices of CDF4.4 (RSW_CN4_L10 / RSW_iCN4_L10 / RSW_CD4_L10 / RSW_iCD4_L10) and of
   CDF2.6 / CDF2.8 with bc 'n', 'd' and 'z' (RSW_L{N,D,Z}{6,8}_L10 and their inverses),
   cuWaveletCompute.cuh:94-137, 150-177, 799-845 */
static const double CN4_L10[25] = {
    2.125, 1.6875, 0.5, -0.6875, -1.625,  -1.625, -0.6875, 0.5, 1.6875, 2.125,  1.0, 0, -2.0, 0, 1.0,
    0.353553390593274, -0.618718433538229, 0.353553390593274, -0.088388347648318, 0,
    0, -0.088388347648318, 0.353553390593274, -0.618718433538229, 0.353553390593274};
static const double ICN4_L10[25] = {
    0.34375, 0.15625, 0.25, 0.773398041922786, -0.066291260736239,
    0.3125, 0.1875, 0, -1.016465997955662, 0.309359216769115,
    0.25, 0.25, -0.25, 0.353553390593274, 0.353553390593274,
    0.1875, 0.3125, 0, 0.309359216769115, -1.016465997955662,
    0.15625, 0.34375, 0.25, -0.066291260736239, 0.773398041922786};
static const double CD4_L10[25] = {
    2.05078125, 0, 0, 0, 0,  0, 0, 0, 0, 2.05078125,
    0.734375, -0.1484375, -0.46875, -0.1484375, 0.734375,
    0.353553390593274, -0.441941738241592, 0.353553390593274, -0.088388347648318, 0,
    0, -0.088388347648318, 0.353553390593274, -0.441941738241592, 0.353553390593274};
static const double ICD4_L10[25] = {
    0.125, 0, 0, 0, 0,
    0.25, 0.125, -1.0, -2.077126169735483, 0.751300955010707,
    0.21875, 0.21875, -1.5, 0.419844651329513, 0.419844651329513,
    0.125, 0.25, -1.0, 0.751300955010707, -2.077126169735483,
    0, 0.125, 0, 0, 0};
static const double LN6_L10[25] = {
    0.8671875, 1.265625, 0.5, -0.265625, -0.3671875,  -0.3671875, -0.265625, 0.5, 1.265625, 0.8671875,
    -0.5, 0, 1.0, 0, -0.5,
    -0.353553390593274, 0.707106781186547, -0.353553390593274, 0, 0,
    0, 0, -0.353553390593274, 0.707106781186547, -0.353553390593274};
static const double ILN6_L10[25] = {
    0.5, 0, -0.5, -0.894932019939224, 0.187825238752677,
    0.375, 0.125, 0, 0.789970857106846, -0.082864075920299,
    0.25, 0.25, 0.5, -0.353553390593274, -0.353553390593274,
    0.125, 0.375, 0, -0.082864075920299, 0.789970857106846,
    0, 0.5, -0.5, 0.187825238752677, -0.894932019939224};
static const double LZ6_L10[25] = {
    0.8671875, 0.6328125, 0.25, -0.1328125, -0.3671875,  -0.3671875, -0.1328125, 0.25, 0.6328125, 0.8671875,
    -1.0, 0, 1.0, 0, -1.0,
    -0.707106781186547, 0.707106781186547, -0.353553390593274, 0, 0,
    0, 0, -0.353553390593274, 0.707106781186547, -0.707106781186547};
static const double ILZ6_L10[25] = {
    0.5, 0, -0.25, -0.447466009969612, 0.093912619376338,
    0.75, 0.25, 0, 0.789970857106846, -0.082864075920299,
    0.5, 0.5, 0.5, -0.353553390593274, -0.353553390593274,
    0.25, 0.75, 0, -0.082864075920299, 0.789970857106846,
    0, 0.5, -0.25, 0.093912619376338, -0.447466009969612};
static const double LD6_L10[25] = {
    2.0, 0, 0, 0, 0,  0, 0, 0, 0, 2.0,
    -0.69140625, 0.3828125, 0.6171875, 0.3828125, -0.69140625,
    -0.353553390593274, 0.707106781186547, -0.353553390593274, 0, 0,
    0, 0, -0.353553390593274, 0.707106781186547, -0.353553390593274};
static const double ILD6_L10[25] = {
    0.5, 0, 0, 0, 0,
    0.375, 0.125, 0.5, 1.143524247700120, -0.270689314672975,
    0.25, 0.25, 1.0, -0.541378629345950, -0.541378629345950,
    0.125, 0.375, 0.5, -0.270689314672975, 1.143524247700120,
    0, 0.5, 0, 0, 0};
static const double LN8_L10[25] = {
    0.85009765625, 1.2998046875, 0.5, -0.2998046875, -0.35009765625,
    -0.35009765625, -0.2998046875, 0.5, 1.2998046875, 0.85009765625,
    -0.5, 0, 1.0, 0, -0.5,
    -0.353553390593274, 0.707106781186548, -0.353553390593274, 0, 0,
    0, 0, -0.353553390593274, 0.707106781186548, -0.353553390593274};
static const double ILN8_L10[25] = {
    0.5, 0, -0.5, -0.919100708749311, 0.211993927562764,
    0.375, 0.125, 0, 0.777886512701802, -0.070779731515255,
    0.25, 0.25, 0.5, -0.353553390593274, -0.353553390593274,
    0.125, 0.375, 0, -0.070779731515255, 0.777886512701803,
    0, 0.5, -0.5, 0.211993927562764, -0.919100708749311};
static const double LD8_L10[25] = {
    0.905622728168965, 0, 0, 0, 0,  0, 0, 0, 0, 0.905622728168965,
    -0.443145751953125, 0.39990234375, 0.60009765625, 0.39990234375, -0.443145751953125,
    -0.353553390593274, 0.707106781186548, -0.353553390593274, 0, 0,
    0, 0, -0.353553390593274, 0.707106781186548, -0.353553390593274};
static const double ILD8_L10[25] = {
    0.5, 0, 0, 0, 0,
    0.375, 0.125, 0.5, 1.131439903295076, -0.282773659078019,
    0.25, 0.25, 1.0, -0.565547318156037, -0.565547318156038,
    0.125, 0.375, 0.5, -0.282773659078019, 1.131439903295076,
    0, 0.5, 0, 0, 0};
static const double LZ8_L10[25] = {
    0.85009765625, 0.64990234375, 0.25, -0.14990234375, -0.35009765625,
    -0.35009765625, -0.14990234375, 0.25, 0.64990234375, 0.85009765625,
    -1.0, 0, 1.0, 0, -1.0,
    -0.707106781186548, 0.707106781186548, -0.353553390593274, 0, 0,
    0, 0, -0.353553390593274, 0.707106781186548, -0.707106781186548};
static const double ILZ8_L10[25] = {
    0.5, 0, -0.25, -0.459550354374656, 0.105996963781382,
    0.75, 0.25, 0, 0.777886512701802, -0.070779731515255,
    0.5, 0.5, 0.5, -0.353553390593274, -0.353553390593274,
    0.25, 0.75, 0, -0.070779731515255, 0.777886512701803,
    0, 0.5, -0.25, 0.105996963781382, -0.459550354374656};

#define IS_C4(w) ((w) == OR_CDF4_6 || (w) == OR_CDF4_4)
#define IS_L2(w) ((w) == OR_CDF2_6 || (w) == OR_CDF2_8)

/* The short families (cuWaveletCompute.cuh:1397-1556; registered at cuWHHDForward.cu:998-1080).
   CDF2.0: CDF2.x's predict alone, no update, the detail's scale negated, CDF2.6's boundary rules
   (cuUpdateCdf20_ad / _ad_i); CDF1.1: the Haar step, d - a then a + d/2 (cuUpdateCdf11_ad / _ad_i);
   CDF1.7: the Haar predict and a 7-tap update, CDF3.5's boundary rules (cuUpdateCdf17_ad / _ad_i). */
#define IS_SHORT(w) ((w) == OR_CDF2_0 || (w) == OR_CDF1_1 || (w) == OR_CDF1_7)
static const double T1_FP = -1.0, T1_FU = 0.5;
static const double T1_SCL[2] = {SQ2, 1.0 / SQ2};
static const double T7_FU[7] = {-0.002441406250000, 0.021484375000000, -0.098144531250000, 0.5,
                                0.098144531250000, -0.021484375000000, 0.002441406250000};
static const double T7_SCL[2] = {SQ2, -1.0 / SQ2};
static const double B20_L10[25] = {
    2.0, 0, 0, 0, 0,
    0, 0, 0, 0, 2.0,
    0.5, 0, -1.0, 0, 0.5,
    0.353553390593274, -0.707106781186547, 0.353553390593274, 0, 0,
    0, 0, 0.353553390593274, -0.707106781186547, 0.353553390593274};
static const double IB20_L10[25] = {
    0.5, 0, 0, 0, 0,
    0.375, 0.125, -0.5, -1.414213562373095, 0,
    0.25, 0.25, -1.0, 0, 0,
    0.125, 0.375, -0.5, 0, -1.414213562373095,
    0, 0.5, 0, 0, 0};
static const double B11_L10[16] = {
    0.5, 0.5, 0.5, 0.5,
    -0.5, -0.5, 0.5, 0.5,
    -0.707106781186548, 0.707106781186548, 0, 0,
    0, 0, -0.707106781186548, 0.707106781186548};
static const double IB11_L10[16] = {
    0.5, -0.5, -0.707106781186547, 0,
    0.5, -0.5, 0.707106781186547, 0,
    0.5, 0.5, 0, -0.707106781186547,
    0.5, 0.5, 0, 0.707106781186547};
static const double TN7_L10[16] = {
    0.5, 0.5, 0.5, 0.5,
    0.691406250000000, 0.308593750000000, -0.308593750000000, -0.691406250000000,
    0.707106781186548, -0.707106781186548, 0, 0,
    0, 0, 0.707106781186548, -0.707106781186548};
static const double ITN7_L10[16] = {
    0.5, 0.5, 0.571762123850060, -0.135344657336488,
    0.5, 0.5, -0.842451438523035, -0.135344657336488,
    0.5, -0.5, 0.135344657336488, 0.842451438523035,
    0.5, -0.5, 0.135344657336488, -0.571762123850060};
static const double TD7_L10[16] = {
    0.308593750000000, 0.691406250000000, 0.691406250000000, 0.308593750000000,
    0.5, 0.5, -0.5, -0.5,
    0.707106781186548, -0.707106781186548, 0, 0,
    0, 0, 0.707106781186548, -0.707106781186548};
static const double ITD7_L10[16] = {
    0.5, 0.5, 0.842451438523035, -0.135344657336488,
    0.5, 0.5, -0.571762123850060, -0.135344657336488,
    0.5, -0.5, 0.135344657336488, 0.571762123850060,
    0.5, -0.5, 0.135344657336488, -0.842451438523035};

/* 'z' is the Dirichlet-with-spacing alias: the CDF3.x wavelets treat it as 'd', the CDF4.x ones as
   'n' (cuWHHDForward.cu:760-765, 886-891, 970-975); CDF2.6 / CDF2.8 have their own 'z' rule
   (cuWHHDForward.cu:802-828, cuWT_CDF2_6_z) */
static char norm_bc(int wavelet, char bc) {
    if (bc == 'z' && !IS_L2(wavelet)) return IS_Q3(wavelet) ? 'd' : 'n';
    return bc;
}

static const double* base_matrix(int wavelet, char bc, int forward) {
    if (wavelet == OR_CDF2_0) return forward ? B20_L10 : IB20_L10;
    if (wavelet == OR_CDF1_1) return forward ? B11_L10 : IB11_L10;
    if (wavelet == OR_CDF1_7) {
        if (bc == 'n') return forward ? TN7_L10 : ITN7_L10;
        return forward ? TD7_L10 : ITD7_L10;
    }
    if (wavelet == OR_CDF3_5) {
        if (bc == 'n') return forward ? QN5_L10 : IQN5_L10;
        return forward ? QD5_L10 : IQD5_L10;
    }
    if (wavelet == OR_CDF3_7) {
        if (bc == 'n') return forward ? QN7_L10 : IQN7_L10;
        return forward ? QD7_L10 : IQD7_L10;
    }
    if (wavelet == OR_CDF4_4) {
        if (bc == 'n') return forward ? CN4_L10 : ICN4_L10;
        return forward ? CD4_L10 : ICD4_L10;
    }
    if (wavelet == OR_CDF2_6) {
        if (bc == 'n') return forward ? LN6_L10 : ILN6_L10;
        if (bc == 'z') return forward ? LZ6_L10 : ILZ6_L10;
        return forward ? LD6_L10 : ILD6_L10;
    }
    if (wavelet == OR_CDF2_8) {
        if (bc == 'n') return forward ? LN8_L10 : ILN8_L10;
        if (bc == 'z') return forward ? LZ8_L10 : ILZ8_L10;
        return forward ? LD8_L10 : ILD8_L10;
    }
    if (bc == 'n') return forward ? CN6_L10 : ICN6_L10;
    return forward ? CD6_L10 : ICD6_L10;
}

/* -------------------------------------------------------- boundary reflection rules ---- */
/* Forward: pair k reads samples 2k (a) and 2k+1 (d) of a level of even length L (+1 if odd).
   CDF3.7: half-sample symmetric about -1/2 and L-1/2; 'd' negates reflected samples
           (cuWaveletCompute.cuh:180-228, cuWT_CDF3_5_n/_d).
   CDF4.6: whole-sample symmetric about 0 and L; 'd' negates reflected samples except the
           boundary sample itself (cuWaveletCompute.cuh:336-375, cuWT_CDF4_4_n/_d). */
static void fwd_reflect(int wavelet, char bc, int k, int L, int* ai, int* di, double* sa, double* sd) {
    int a = 2 * k, d = 2 * k + 1;
    double s_a = 1.0, s_d = 1.0;
    if (IS_Q3(wavelet) || wavelet == OR_CDF1_1 || wavelet == OR_CDF1_7) {
        if (a < 0) { a = -1 - a; if (bc == 'd') s_a = -1.0; }
        else if (a >= L) { a = 2 * L - 1 - a; if (bc == 'd') s_a = -1.0; }
        if (d < 0) { d = -1 - d; if (bc == 'd') s_d = -1.0; }
        else if (d >= L) { d = 2 * L - 1 - d; if (bc == 'd') s_d = -1.0; }
    } else if (IS_L2(wavelet) && bc == 'd') {
        /* cuWT_CDF2_6_d (cuWaveletCompute.cuh:271-294): a whole-sample reflection of a with no sign,
           d reflected separately with a negative sign */
        if (a < 0) a = -a;
        else if (a > L) a = 2 * L - a;
        if (d < 0) { d = -d; s_d = -1.0; }
        else if (d >= L) { d = 2 * L - d; s_d = -1.0; }
    } else {
        int a_orig = a;
        if (a < 0) { a = -a; d = -d; if (bc == 'd') { s_a = -1.0; s_d = -1.0; } }
        else if (a >= L) { a = 2 * L - a; d = 2 * L - d; if (bc == 'd') { s_a = -1.0; s_d = -1.0; } }
        if (bc == 'd' && a_orig == L) s_a = 1.0;
        /* cuWT_CDF2_6_z (:296-311): the boundary samples count twice */
        if (bc == 'z' && (a == 0 || a == L)) s_a = 2.0;
    }
    if (d < 0) d = 0; /* cuWHHDForward.cu:52 clamps the odd index */
    *ai = a; *di = d; *sa = s_a; *sd = s_d;
}

/* Inverse: index k reads approximation a[k] (length L+ext) and detail d[k] (length L).
   CDF3.7: cuWaveletCompute.cuh:600-631 (cuWT_CDF3_5_n_i/_d_i); CDF4.6: :716-752. */
static void inv_reflect(int wavelet, char bc, int k, int L, int* ai, int* di, double* sa, double* sd) {
    int a = k, d = k;
    double s_a = 1.0, s_d = 1.0;
    if (IS_Q3(wavelet) || wavelet == OR_CDF1_1 || wavelet == OR_CDF1_7) {
        if (a < 0) { a = -1 - a; if (bc == 'n') s_d = -1.0; else s_a = -1.0; }
        else if (a >= L) { a = 2 * L - 1 - a; if (bc == 'n') s_d = -1.0; else s_a = -1.0; }
        d = a;
    } else if (bc == 'n' || bc == 'z') {
        /* cuWT_CDF2_6_z_i (:684-699): the sign is 2 at the two boundary indices, read before the
           reflection */
        if (bc == 'z' && (a == 0 || a == L)) s_a = 2.0;
        if (a < 0) { a = -a; d = -d - 1; }
        else if (a >= L) { a = 2 * L - a; d = 2 * L - d - 1; }
    } else if (IS_L2(wavelet)) {
        /* cuWT_CDF2_6_d_i (:668-683) */
        if (a < 0) { a = -a; d = -d - 1; s_d = -1.0; }
        else if (a >= L) { a = 2 * L - a; d = 2 * L - d - 1; s_d = -1.0; }
    } else {
        if (a < 0) { a = -a; d = -d - 1; s_d = -1.0; s_a = -1.0; }
        else if (a >= L) { d = 2 * L - d - 1; s_d = -1.0; }
        if (a > L) { a = 2 * L - a; s_a = -1.0; }
    }
    *ai = a; *di = d; *sa = s_a; *sd = s_d;
}

/* ------------------------------------------------------------ one lifting level ---- */
/* forward level: x (length L+ext) -> a (M = L/2+ext), d (L/2).  cuWHHDForward.cu:37-73 with the
   step functions cuUpdateCdf37_ad (cuWaveletCompute.cuh:876-900) / cuUpdateCdf46_ad (:925-942) */
static void fwd_level(const double* x, int L, int ext, int wavelet, char bc, double* a_out, double* d_out,
                      double* work) {
    int M = L / 2 + ext;
    int K0 = -HALO, K1 = M + HALO, W = K1 - K0;
    double* A0 = work;
    double* D0 = A0 + W;
    double* A1 = D0 + W;
    double* D1 = A1 + W;
    int n_in = L + ext;
#define IX(k) ((k) - K0)
    for (int k = K0; k < K1; ++k) {
        int ai, di; double sa, sd;
        fwd_reflect(wavelet, bc, k, L, &ai, &di, &sa, &sd);
        A0[IX(k)] = (ai >= 0 && ai < n_in) ? sa * x[ai] : 0.0;
        D0[IX(k)] = (di >= 0 && di < n_in) ? sd * x[di] : 0.0;
    }
    for (int k = K0; k < K1; ++k) { A1[IX(k)] = 0.0; D1[IX(k)] = 0.0; }
    if (wavelet == OR_CDF2_0) {
        /* the predict on the raw samples (no reflection sign: it reads no sample outside the line) */
        for (int k = 0; k < L / 2; ++k)
            d_out[k] = (x[2 * k + 1] + L6_FP[0] * x[2 * k] + L6_FP[1] * x[2 * k + 2]) * -L6_SCL[1];
        for (int k = 0; k < M; ++k) a_out[k] = x[2 * k] * L6_SCL[0];
    } else if (wavelet == OR_CDF1_1 || wavelet == OR_CDF1_7) {
        for (int k = K0; k < K1; ++k) D1[IX(k)] = D0[IX(k)] + T1_FP * A0[IX(k)];
        for (int k = 0; k < M; ++k) {
            double s = A0[IX(k)];
            if (wavelet == OR_CDF1_1) s += T1_FU * D1[IX(k)];
            else
                for (int j = -3; j <= 3; ++j) s += T7_FU[3 - j] * D1[IX(k + j)];
            a_out[k] = s * (wavelet == OR_CDF1_1 ? T1_SCL[0] : T7_SCL[0]);
        }
        for (int k = 0; k < L / 2; ++k) d_out[k] = D1[IX(k)] * (wavelet == OR_CDF1_1 ? T1_SCL[1] : T7_SCL[1]);
    } else if (IS_L2(wavelet)) {
        /* predict with the signed approximations, then the detail's own sign, then the update;
           the approximation's sign is divided out at the end (cuUpdateCdf26_ad / cuUpdateCdf28_ad) */
        const double* fu = wavelet == OR_CDF2_6 ? L6_FU : L8_FU;
        const int nt = wavelet == OR_CDF2_6 ? 6 : 8, lo = nt / 2; /* taps k - lo .. k + lo - 1 */
        double* SA = D1 + W;
        double* SD = SA + W;
        for (int k = K0; k < K1; ++k) {
            int ai, di; double sa, sd;
            fwd_reflect(wavelet, bc, k, L, &ai, &di, &sa, &sd);
            D0[IX(k)] = (di >= 0 && di < n_in) ? x[di] : 0.0; /* the detail's sign comes after the predict */
            SA[IX(k)] = sa; SD[IX(k)] = sd;
        }
        for (int k = K0; k < K1 - 1; ++k)
            D1[IX(k)] = (D0[IX(k)] + L6_FP[0] * A0[IX(k)] + L6_FP[1] * A0[IX(k + 1)]) * SD[IX(k)];
        for (int k = 0; k < M; ++k) {
            double s = A0[IX(k)];
            for (int t = 0; t < nt; ++t) s += fu[nt - 1 - t] * D1[IX(k - lo + t)];
            a_out[k] = s * L6_SCL[0] / SA[IX(k)];
        }
        for (int k = 0; k < L / 2; ++k) d_out[k] = D1[IX(k)] * L6_SCL[1];
    } else if (IS_Q3(wavelet)) {
        const double* fu2 = wavelet == OR_CDF3_5 ? Q5_FU2 : Q7_FU2;
        const int hw = wavelet == OR_CDF3_5 ? 2 : 3;
        for (int k = K0 + 1; k < K1; ++k) A1[IX(k)] = A0[IX(k)] + Q5_FU1 * D0[IX(k - 1)];
        for (int k = K0 + 1; k < K1 - 1; ++k)
            D1[IX(k)] = D0[IX(k)] + Q5_FP[0] * A1[IX(k + 1)] + Q5_FP[1] * A1[IX(k)];
        for (int k = 0; k < M; ++k) {
            double s = A1[IX(k)];
            for (int t = -hw; t <= hw; ++t) s += fu2[hw - t] * D1[IX(k + t)];
            a_out[k] = s * Q5_SCL[0];
        }
        for (int k = 0; k < L / 2; ++k) d_out[k] = D1[IX(k)] * Q5_SCL[1];
    } else {
        for (int k = K0 + 1; k < K1; ++k)
            A1[IX(k)] = A0[IX(k)] + C4_FU1[1] * D0[IX(k - 1)] + C4_FU1[0] * D0[IX(k)];
        for (int k = K0 + 1; k < K1 - 1; ++k)
            D1[IX(k)] = D0[IX(k)] + C4_FP[1] * A1[IX(k)] + C4_FP[0] * A1[IX(k + 1)];
        for (int k = 0; k < M; ++k) {
            double s = A1[IX(k)];
            if (wavelet == OR_CDF4_4)
                s += C4_FU2[3] * D1[IX(k - 2)] + C4_FU2[2] * D1[IX(k - 1)] + C4_FU2[1] * D1[IX(k)] +
                     C4_FU2[0] * D1[IX(k + 1)];
            else
                s += C6_FU2[5] * D1[IX(k - 3)] + C6_FU2[4] * D1[IX(k - 2)] + C6_FU2[3] * D1[IX(k - 1)] +
                     C6_FU2[2] * D1[IX(k)] + C6_FU2[1] * D1[IX(k + 1)] + C6_FU2[0] * D1[IX(k + 2)];
            a_out[k] = s * C4_SCL[0];
        }
        for (int k = 0; k < L / 2; ++k) d_out[k] = D1[IX(k)] * C4_SCL[1];
    }
#undef IX
}

/* inverse level: a (L+ext), d (L) -> x (2L+ext).  cuWHHDForward.cu:402-440 with the step functions
   cuUpdateCdf37_ad_i (cuWaveletCompute.cuh:944-964) / cuUpdateCdf46_ad_i (:983-1002).  The CDF4.6
   inverse re-applies the reflection signs between its steps exactly as the reference does. */
static void inv_level(const double* a, const double* d, int L, int ext, int wavelet, char bc, double* x,
                      double* work) {
    int NA = L + ext;
    int K0 = -HALO, K1 = NA + HALO, W = K1 - K0;
    double* A = work;
    double* D = A + W;
    double* SA = D + W;
    double* SD = SA + W;
    double* T = SD + W;
#define IX(k) ((k) - K0)
    for (int k = K0; k < K1; ++k) {
        int ai, di; double sa, sd;
        inv_reflect(wavelet, bc, k, L, &ai, &di, &sa, &sd);
        A[IX(k)] = (ai >= 0 && ai < NA) ? a[ai] : 0.0;
        D[IX(k)] = (di >= 0 && di < L) ? d[di] : 0.0;
        SA[IX(k)] = sa; SD[IX(k)] = sd;
    }
    if (wavelet == OR_CDF2_0) {
        for (int k = 0; k < NA; ++k) x[2 * k] = a[k] * L6_SCL[1];
        for (int k = 0; k < L; ++k)
            x[2 * k + 1] = -d[k] * L6_SCL[0] - (L6_FP[1] * x[2 * k] + L6_FP[0] * x[2 * k + 2]);
    } else if (wavelet == OR_CDF1_1) {
        for (int k = 0; k < L; ++k) {
            const double dd = d[k] * T1_SCL[0];
            const double aa = a[k] * T1_SCL[1] - T1_FU * dd;
            x[2 * k] = aa;
            x[2 * k + 1] = dd - T1_FP * aa;
        }
    } else if (wavelet == OR_CDF1_7) {
        for (int k = K0; k < K1; ++k) {
            D[IX(k)] = SD[IX(k)] * D[IX(k)] / T7_SCL[1];
            A[IX(k)] = SA[IX(k)] * A[IX(k)] / T7_SCL[0];
        }
        for (int k = 0; k < L; ++k) {
            double t = A[IX(k)];
            for (int j = -3; j <= 3; ++j) t -= T7_FU[3 - j] * D[IX(k + j)];
            x[2 * k] = t;
            x[2 * k + 1] = D[IX(k)] - T1_FP * t;
        }
    } else if (IS_L2(wavelet)) {
        const double* fu = wavelet == OR_CDF2_6 ? L6_FU : L8_FU;
        const int nt = wavelet == OR_CDF2_6 ? 6 : 8, lo = nt / 2;
        for (int k = K0; k < K1; ++k) {
            D[IX(k)] = SD[IX(k)] * D[IX(k)] * L6_SCL[0];
            A[IX(k)] = SA[IX(k)] * A[IX(k)] * L6_SCL[1];
        }
        for (int k = K0 + lo; k < K1 - lo; ++k) {
            double t = A[IX(k)];
            for (int j = 0; j < nt; ++j) t -= fu[nt - 1 - j] * D[IX(k - lo + j)];
            T[IX(k)] = t;
        }
        for (int k = 0; k < NA; ++k) x[2 * k] = T[IX(k)] / SA[IX(k)];
        for (int k = 0; k < L; ++k) x[2 * k + 1] = D[IX(k)] - (L6_FP[1] * T[IX(k)] + L6_FP[0] * T[IX(k + 1)]);
    } else if (IS_Q3(wavelet)) {
        const double* fu2 = wavelet == OR_CDF3_5 ? Q5_FU2 : Q7_FU2;
        const int hw = wavelet == OR_CDF3_5 ? 2 : 3;
        for (int k = K0; k < K1; ++k) {
            A[IX(k)] = SA[IX(k)] * A[IX(k)] * Q5_SCL[1];
            D[IX(k)] = SD[IX(k)] * D[IX(k)] * Q5_SCL[0];
        }
        for (int k = K0 + 3; k < K1 - 3; ++k) {
            double s = 0.0;
            for (int t = -hw; t <= hw; ++t) s += fu2[hw - t] * D[IX(k + t)];
            T[IX(k)] = A[IX(k)] - s;
        }
        for (int k = K0 + 3; k < K1 - 4; ++k) D[IX(k)] = D[IX(k)] - (Q5_FP[1] * T[IX(k)] + Q5_FP[0] * T[IX(k + 1)]);
        for (int k = 0; k < NA; ++k) x[2 * k] = T[IX(k)] - Q5_FU1 * D[IX(k - 1)];
        for (int k = 0; k < L; ++k) x[2 * k + 1] = D[IX(k)];
    } else {
        for (int k = K0; k < K1; ++k) {
            D[IX(k)] = SD[IX(k)] * D[IX(k)] * C4_SCL_INV[1];
            A[IX(k)] = SA[IX(k)] * A[IX(k)] * C4_SCL_INV[0];
        }
        for (int k = K0 + 3; k < K1 - 2; ++k) {
            double s = wavelet == OR_CDF4_4
                           ? C4_FU2[3] * D[IX(k - 2)] + C4_FU2[2] * D[IX(k - 1)] + C4_FU2[1] * D[IX(k)] +
                                 C4_FU2[0] * D[IX(k + 1)]
                           : C6_FU2[5] * D[IX(k - 3)] + C6_FU2[4] * D[IX(k - 2)] + C6_FU2[3] * D[IX(k - 1)] +
                                 C6_FU2[2] * D[IX(k)] + C6_FU2[1] * D[IX(k + 1)] + C6_FU2[0] * D[IX(k + 2)];
            T[IX(k)] = SA[IX(k)] * (A[IX(k)] - s); /* A3 = sign_a * A2 */
        }
        for (int k = K0; k < K1; ++k) D[IX(k)] = SD[IX(k)] * D[IX(k)]; /* D2 = sign_d * D1 */
        for (int k = K0 + 3; k < K1 - 3; ++k)
            D[IX(k)] = SD[IX(k)] * (D[IX(k)] - (C4_FP[1] * T[IX(k)] + C4_FP[0] * T[IX(k + 1)]));
        for (int k = 0; k < NA; ++k) x[2 * k] = T[IX(k)] - (C4_FU1[1] * D[IX(k - 1)] + C4_FU1[0] * D[IX(k)]);
        for (int k = 0; k < L; ++k) x[2 * k + 1] = D[IX(k)];
    }
#undef IX
}

/* ----------------------------------------------------------------- full 1D line ---- */
int or_dwt_line(double* line, int n, int levels, int wavelet, char bc, int forward) {
    if (!IS_Q3(wavelet) && !IS_C4(wavelet) && !IS_L2(wavelet) && !IS_SHORT(wavelet)) return 2;
    /* the short families register 'n' and 'd' only (cuWHHDForward.cu:998-1080) */
    if (IS_SHORT(wavelet) && bc != 'n' && bc != 'd') return 2;
    bc = norm_bc(wavelet, bc);
    if (bc != 'n' && bc != 'd' && !(bc == 'z' && IS_L2(wavelet))) return 2;
    int ext = n & 1;
    if (levels < 2 || (1 << levels) != n - ext) return 1;
    /* the CDF4.4 and CDF2.x base matrices act on 5 coefficients: whole-sample lines of 2^L + 1 */
    if ((wavelet == OR_CDF4_4 || IS_L2(wavelet) || wavelet == OR_CDF2_0) && !ext) return 1;
    if ((wavelet == OR_CDF1_1 || wavelet == OR_CDF1_7) && ext) return 1;
    int nb = 4 + ext;
    double* buf = (double*)malloc(sizeof(double) * (size_t)(2 * n + 16));
    double* tmp = buf + n + 8;
    double* work = (double*)malloc(sizeof(double) * (size_t)(6 * (n + 2 * HALO + 8)));
    const double* mat = base_matrix(wavelet, bc, forward);
    memcpy(buf, line, sizeof(double) * n);
    if (forward) {
        for (int l = levels - 1; l > 1; --l) {
            int L = 1 << (l + 1);
            int M = L / 2 + ext;
            fwd_level(buf, L, ext, wavelet, bc, tmp, tmp + M, work);
            memcpy(buf, tmp, sizeof(double) * (L + ext));
        }
        for (int i = 0; i < nb; ++i) {
            double s = 0.0;
            for (int j = 0; j < nb; ++j) s += mat[i * nb + j] * buf[j];
            tmp[i] = s;
        }
        memcpy(buf, tmp, sizeof(double) * nb);
    } else {
        for (int i = 0; i < nb; ++i) {
            double s = 0.0;
            for (int j = 0; j < nb; ++j) s += mat[i * nb + j] * buf[j];
            tmp[i] = s;
        }
        memcpy(buf, tmp, sizeof(double) * nb);
        for (int l = 2; l < levels; ++l) {
            int L = 1 << l;
            inv_level(buf, buf + L + ext, L, ext, wavelet, bc, tmp, work);
            memcpy(buf, tmp, sizeof(double) * (2 * L + ext));
        }
    }
    memcpy(line, buf, sizeof(double) * n);
    free(work);
    free(buf);
    return 0;
}

int or_dwt_axis(double* arr, int DX, int DY, int DZ, int levels, char axis, int wavelet, char bc, int forward) {
    int n, nlines;
    long stride;
    if (axis == 'y' || axis == 'Y') { n = DY; nlines = DX * DZ; stride = 1; }
    else if (axis == 'x' || axis == 'X') { n = DX; nlines = DY * DZ; stride = DY; }
    else { n = DZ; nlines = DX * DY; stride = (long)DX * DY; }
    int ext = n & 1;
    if (levels < 2 || (1 << levels) != n - ext) return 1;
    int err = 0;
#pragma omp parallel for schedule(static) reduction(| : err)
    for (int li = 0; li < nlines; ++li) {
        long base;
        if (axis == 'y' || axis == 'Y') { int x = li % DX, z = li / DX; base = (long)x * DY + (long)z * DX * DY; }
        else if (axis == 'x' || axis == 'X') { int y = li % DY, z = li / DY; base = y + (long)z * DX * DY; }
        else { int y = li % DY, x = li / DY; base = y + (long)x * DY; }
        double* line = (double*)malloc(sizeof(double) * (size_t)n);
        for (int i = 0; i < n; ++i) line[i] = arr[base + i * stride];
        err |= or_dwt_line(line, n, levels, wavelet, bc, forward);
        for (int i = 0; i < n; ++i) arr[base + i * stride] = line[i];
        free(line);
    }
    return err;
}

/* diag(B B^T): the squared norms of the synthesis basis functions.  The reference inverse-
   transforms the identity, multiplies by its transpose and keeps the diagonal band 0
   (cuGetInnerProduct.cu:92-126, :11-22). */
int or_ip_diag(double* out, int dim, int wavelet, char bc) {
    int levels = 0;
    while ((2 << levels) <= dim) ++levels;
    int err = 0;
#pragma omp parallel for schedule(static) reduction(| : err)
    for (int i = 0; i < dim; ++i) {
        double* e = (double*)calloc((size_t)dim, sizeof(double));
        e[i] = 1.0;
        err |= or_dwt_line(e, dim, levels, wavelet, bc, 0);
        double s = 0.0;
        for (int j = 0; j < dim; ++j) s += e[j] * e[j];
        out[i] = s;
        free(e);
    }
    return err;
}

static int ilog2(int n) {
    int l = 0;
    while ((1 << (l + 1)) <= n) ++l;
    return l;
}
static int bitlen(int v) {
    int b = 0;
    while (v > 0) { ++b; v >>= 1; }
    return b;
}

/* ------------------------------------------------------------- local projection ---- */
/* cuProjectLocal_q_3d_dq_ccc (cuDivLocalProject3D.cu:4013-4246): wall bc 'n' gives the div
   wavelet bc 'd'.  Coefficient index (x,y,z) in [0,n)^3 reads xv(x+1,y,z), yv(x,y+1,z),
   zv(x,y,z+1) and writes qx(x,y+1,z+1), qy(x+1,y,z+1), qz(x+1,y+1,z).  Interior: q = (s x v)/|s|^2
   with s_i = 4/(dx_i 2^j_i); faces: one-component inner-product ratios; edges/corner: 0. */
int or_project3d(double* qx, double* qy, double* qz, const double* xv, const double* yv, const double* zv,
                 int nx, int ny, int nz, double dx, double dy, double dz) {
    int Lx = ilog2(nx), Ly = ilog2(ny), Lz = ilog2(nz);
    if ((1 << Lx) != nx || (1 << Ly) != ny || (1 << Lz) != nz) return 1;
    double* ipbx = (double*)malloc(sizeof(double) * (nx + 1));
    double* ipby = (double*)malloc(sizeof(double) * (ny + 1));
    double* ipbz = (double*)malloc(sizeof(double) * (nz + 1));
    double* ippx = (double*)malloc(sizeof(double) * nx);
    double* ippy = (double*)malloc(sizeof(double) * ny);
    double* ippz = (double*)malloc(sizeof(double) * nz);
    or_ip_diag(ipbx, nx + 1, OR_CDF4_6, 'd');
    or_ip_diag(ipby, ny + 1, OR_CDF4_6, 'd');
    or_ip_diag(ipbz, nz + 1, OR_CDF4_6, 'd');
    or_ip_diag(ippx, nx, OR_CDF3_7, 'n');
    or_ip_diag(ippy, ny, OR_CDF3_7, 'n');
    or_ip_diag(ippz, nz, OR_CDF3_7, 'n');
    long sqx = (long)(nx + 1) * ny * (nz + 1), sqy = (long)(nx + 1) * ny * (nz + 1);
    memset(qx, 0, sizeof(double) * (size_t)nx * (ny + 1) * (nz + 1));
    memset(qy, 0, sizeof(double) * (size_t)sqy);
    memset(qz, 0, sizeof(double) * (size_t)(nx + 1) * (ny + 1) * nz);
    (void)sqx;
    double dxi = 1.0 / dx, dyi = 1.0 / dy, dzi = 1.0 / dz;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y) {
                int jx = Lx - bitlen(x) + 1, jy = Ly - bitlen(y) + 1, jz = Lz - bitlen(z) + 1;
                double sx = 4.0 * dxi / ((double)(1 << jx) + EPS12);
                double sy = 4.0 * dyi / ((double)(1 << jy) + EPS12);
                double sz = 4.0 * dzi / ((double)(1 << jz) + EPS12);
                double ip0x = ippx[x], ip1x = ipbx[x + 1];
                double ip0y = ippy[y], ip1y = ipby[y + 1];
                double ip0z = ippz[z], ip1z = ipbz[z + 1];
                double xin = xv[y + (long)(x + 1) * ny + (long)z * (nx + 1) * ny];
                double yin = yv[(y + 1) + (long)x * (ny + 1) + (long)z * nx * (ny + 1)];
                double zin = zv[y + (long)x * ny + (long)(z + 1) * nx * ny];
                double sxBxBy = sx * ip0x * ip1y * ip0z, syBxBy = sy * ip1x * ip0y * ip0z;
                double sxBxBz = sx * ip0x * ip0y * ip1z, szBxBz = sz * ip1x * ip0y * ip0z;
                double syByBz = sy * ip0x * ip0y * ip1z, szByBz = sz * ip0x * ip1y * ip0z;
                double sX = 0.0, sY = 0.0, sZ = 0.0;
                if (x > 0 && y > 0 && z > 0) {
                    double inv = 1.0 / (sy * sy + sx * sx + sz * sz);
                    sZ = (sy * xin - sx * yin) * inv;
                    sX = (sz * yin - sy * zin) * inv;
                    sY = (sx * zin - sz * xin) * inv;
                } else if (y > 0 && z > 0 && x == 0) {
                    sX = (yin * szByBz - zin * syByBz) / (sy * syByBz + sz * szByBz + EPS12);
                } else if (x > 0 && z > 0 && y == 0) {
                    sY = (zin * sxBxBz - xin * szBxBz) / (sx * sxBxBz + sz * szBxBz + EPS12);
                } else if (x > 0 && y > 0 && z == 0) {
                    sZ = (xin * syBxBy - yin * sxBxBy) / (sx * sxBxBy + sy * syBxBy + EPS12);
                }
                qx[(y + 1) + (long)x * (ny + 1) + (long)(z + 1) * nx * (ny + 1)] = sX;
                qy[y + (long)(x + 1) * ny + (long)(z + 1) * (nx + 1) * ny] = sY;
                qz[(y + 1) + (long)(x + 1) * (ny + 1) + (long)z * (nx + 1) * (ny + 1)] = sZ;
            }
    free(ipbx); free(ipby); free(ipbz); free(ippx); free(ippy); free(ippz);
    return 0;
}

/* Local projection with Dirichlet domain walls (the recovery's bc 'd': base wavelet CDF4.6 with bc
   'n', projection wavelet CDF3.7 with bc 'd'), cuProjectLocal_q_3d_nq_ccc
   (cuDivLocalProject3D.cu:4474-4877), launched by ProjectLocal_q_ccc (:5271-5308).  Coefficient
   (x, y, z) in [0, n)^3 with the velocity coefficients X = xv(x+1, y, z), Y = yv(x, y+1, z),
   Z = zv(x, y, z+1) and, on a wall plane, the wall-side ones X0 = xv(x, y, z), Y0 = yv(x, y, z),
   Z0 = zv(x, y, z):
   - interior (x, y, z > 0): q = (s x v) / |s|^2 as for bc 'n';
   - a wall plane (one index 0): the wall-normal velocity pair is divided by the scale of the other
     in-plane axis (the reference's cuCalculateP0Val_single, :156-177), which corrects the in-plane
     velocity by the difference of the two times dx_inv_a / n_a; the remaining
     component is the one-component ratio weighted by the inner-product tables;
   - a wall line (two indices 0): two such corrections, the third component 0;
   - the corner: the base potentials from the wall velocities times the spacings.
   Every potential entry with an index 0 along one of its own axes is written by exactly one
   coefficient (the zero entries included), so the result does not depend on the start of q. */
int or_project3d_nq(double* qx, double* qy, double* qz, const double* xv, const double* yv, const double* zv,
                    int nx, int ny, int nz, double dx, double dy, double dz) {
    int Lx = ilog2(nx), Ly = ilog2(ny), Lz = ilog2(nz);
    if ((1 << Lx) != nx || (1 << Ly) != ny || (1 << Lz) != nz) return 1;
    double* ipbx = (double*)malloc(sizeof(double) * (nx + 1));
    double* ipby = (double*)malloc(sizeof(double) * (ny + 1));
    double* ipbz = (double*)malloc(sizeof(double) * (nz + 1));
    double* ippx = (double*)malloc(sizeof(double) * nx);
    double* ippy = (double*)malloc(sizeof(double) * ny);
    double* ippz = (double*)malloc(sizeof(double) * nz);
    or_ip_diag(ipbx, nx + 1, OR_CDF4_6, 'n');
    or_ip_diag(ipby, ny + 1, OR_CDF4_6, 'n');
    or_ip_diag(ipbz, nz + 1, OR_CDF4_6, 'n');
    or_ip_diag(ippx, nx, OR_CDF3_7, 'd');
    or_ip_diag(ippy, ny, OR_CDF3_7, 'd');
    or_ip_diag(ippz, nz, OR_CDF3_7, 'd');
    const double dxi = 1.0 / dx, dyi = 1.0 / dy, dzi = 1.0 / dz;
    /* inverse extent of the domain along each axis, dx_inv / n (the reference's L_inv) */
    const double lx = dxi / nx, ly = dyi / ny, lz = dzi / nz;
    const long pqx = (long)nx * (ny + 1), pqy = (long)(nx + 1) * ny, pqz = (long)(nx + 1) * (ny + 1);
#define QX(X_, Y_, Z_) qx[(Y_) + (long)(X_) * (ny + 1) + (long)(Z_) * pqx]
#define QY(X_, Y_, Z_) qy[(Y_) + (long)(X_) * ny + (long)(Z_) * pqy]
#define QZ(X_, Y_, Z_) qz[(Y_) + (long)(X_) * (ny + 1) + (long)(Z_) * pqz]
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y) {
                int jx = Lx - bitlen(x) + 1, jy = Ly - bitlen(y) + 1, jz = Lz - bitlen(z) + 1;
                double sx = 4.0 * dxi / ((double)(1 << jx) + EPS12);
                double sy = 4.0 * dyi / ((double)(1 << jy) + EPS12);
                double sz = 4.0 * dzi / ((double)(1 << jz) + EPS12);
                double ip0x = ippx[x], ip1x = ipbx[x + 1];
                double ip0y = ippy[y], ip1y = ipby[y + 1];
                double ip0z = ippz[z], ip1z = ipbz[z + 1];
                double X = xv[y + (long)(x + 1) * ny + (long)z * (nx + 1) * ny];
                double Y = yv[(y + 1) + (long)x * (ny + 1) + (long)z * nx * (ny + 1)];
                double Z = zv[y + (long)x * ny + (long)(z + 1) * nx * ny];
                double X0 = xv[y + (long)x * ny + (long)z * (nx + 1) * ny];
                double Y0 = yv[y + (long)x * (ny + 1) + (long)z * nx * (ny + 1)];
                double Z0 = zv[y + (long)x * ny + (long)z * nx * ny];
                double b010 = ip0x * ip1y * ip0z, b100 = ip1x * ip0y * ip0z, b001 = ip0x * ip0y * ip1z;
                double wx = 1.0 / (sy * (sy * b001) + sz * (sz * b010) + EPS12);
                double wy = 1.0 / (sx * (sx * b001) + sz * (sz * b100) + EPS12);
                double wz = 1.0 / (sx * (sx * b010) + sy * (sy * b100) + EPS12);
                double oX = 0.0, oY = 0.0, oZ = 0.0;
                int zx = x == 0, zy = y == 0, zz = z == 0;
                if (!zx && !zy && !zz) {
                    double inv = 1.0 / (sy * sy + sx * sx + sz * sz);
                    oZ = (sy * X - sx * Y) * inv;
                    oX = (sz * Y - sy * Z) * inv;
                    oY = (sx * Z - sz * X) * inv;
                } else if (zz && !zx && !zy) {  /* wall plane z = 0 */
                    double t0 = Z0 / sx, t1 = Z / sx;
                    X += (t1 - t0) * lz;
                    QX(x, y + 1, 0) = 0.0;
                    QY(x + 1, y, 0) = t0;
                    oY = t1;
                    oZ = (X * (sy * b100) - Y * (sx * b010)) * wz;
                } else if (zy && !zx && !zz) {  /* wall plane y = 0 */
                    double t0 = Y0 / sz, t1 = Y / sz;
                    Z += (t1 - t0) * ly;
                    QX(x, 0, z + 1) = t0;
                    QZ(x + 1, 0, z) = 0.0;
                    oX = t1;
                    oY = (Z * (sx * b001) - X * (sz * b100)) * wy;
                } else if (zx && !zy && !zz) {  /* wall plane x = 0 */
                    double t0 = X0 / sy, t1 = X / sy;
                    Y += (t1 - t0) * lx;
                    QZ(0, y + 1, z) = t0;
                    QY(0, y, z + 1) = 0.0;
                    oZ = t1;
                    oX = (Y * (sz * b010) - Z * (sy * b001)) * wx;
                } else if (!zx && zy && zz) {  /* wall line along x */
                    double a0 = Z0 / sx, a1 = Z / sx;
                    double c0 = -Y0 / sx, c1 = -Y / sx;
                    QY(x + 1, 0, 0) = a0;
                    QZ(x + 1, 0, 0) = c0;
                    QX(x, 0, 1) = 0.0;
                    QX(x, 0, 0) = 0.0;
                    QX(x, 1, 0) = 0.0;
                    oY = a1;
                    oZ = c1;
                } else if (zx && !zy && zz) {  /* wall line along y */
                    double a0 = -Z0 / sy, a1 = -Z / sy;
                    double c0 = X0 / sy, c1 = X / sy;
                    QX(0, y + 1, 0) = a0;
                    QZ(0, y + 1, 0) = c0;
                    QY(0, y, 0) = 0.0;
                    QY(1, y, 0) = 0.0;
                    QY(0, y, 1) = 0.0;
                    oX = a1;
                    oZ = c1;
                } else if (zx && zy && !zz) {  /* wall line along z */
                    double a0 = Y0 / sz, a1 = Y / sz;
                    double c0 = -X0 / sz, c1 = -X / sz;
                    QX(0, 0, z + 1) = a0;
                    QY(0, 0, z + 1) = c0;
                    QZ(0, 0, z) = 0.0;
                    QZ(0, 1, z) = 0.0;
                    QZ(1, 0, z) = 0.0;
                    oX = a1;
                    oY = c1;
                } else {  /* corner */
                    double x010 = -Z0 / ly, x001 = Y0 / lz, x011 = x010 + Y / lz;
                    double y001 = -X0 / lz, y101 = -X / lz;
                    QZ(0, 0, 0) = 0.0;
                    QZ(1, 0, 0) = 0.0;
                    QZ(0, 1, 0) = 0.0;
                    QX(0, 0, 0) = 0.0;
                    QX(0, 1, 0) = x010;
                    QX(0, 0, 1) = x001;
                    QY(0, 0, 0) = 0.0;
                    QY(1, 0, 0) = 0.0;
                    QY(0, 0, 1) = y001;
                    oX = x011;
                    oY = y101;
                }
                QX(x, y + 1, z + 1) = oX;
                QY(x + 1, y, z + 1) = oY;
                QZ(x + 1, y + 1, z) = oZ;
            }
#undef QX
#undef QY
#undef QZ
    free(ipbx); free(ipby); free(ipbz); free(ippx); free(ippy); free(ippz);
    return 0;
}

/* cuProjectLocal_q_single (cuDivLocalProject.cu:765-1045): both passes evaluate the same pointwise
   ratio and the neighbour terms are unused, so qz(x,y) = P for 2<=x<=nx, 2<=y<=ny, else 0. */
int or_project2d(double* qz, const double* xv, const double* yv, int nx, int ny, double dx, double dy) {
    int Lx = ilog2(nx), Ly = ilog2(ny);
    if ((1 << Lx) != nx || (1 << Ly) != ny) return 1;
    double* ipbx = (double*)malloc(sizeof(double) * (nx + 1));
    double* ipby = (double*)malloc(sizeof(double) * (ny + 1));
    double* ippx = (double*)malloc(sizeof(double) * nx);
    double* ippy = (double*)malloc(sizeof(double) * ny);
    or_ip_diag(ipbx, nx + 1, OR_CDF4_6, 'd');
    or_ip_diag(ipby, ny + 1, OR_CDF4_6, 'd');
    or_ip_diag(ippx, nx, OR_CDF3_7, 'n');
    or_ip_diag(ippy, ny, OR_CDF3_7, 'n');
    double dxi = 1.0 / dx, dyi = 1.0 / dy;
    for (int x = 0; x <= nx; ++x)
        for (int y = 0; y <= ny; ++y) {
            double val = 0.0;
            if (x >= 2 && y >= 2) {
                int jx = Lx - bitlen(x - 1) + 1, jy = Ly - bitlen(y - 1) + 1;
                double sx = 4.0 * dxi / ((double)(1 << jx) + EPS12);
                double sy = 4.0 * dyi / ((double)(1 << jy) + EPS12);
                double ip0x = ippx[x - 1], ip1x = ipbx[x], ip0y = ippy[y - 1], ip1y = ipby[y];
                double xin = xv[(y - 1) + (long)x * ny];
                double yin = yv[y + (long)(x - 1) * (ny + 1)];
                double mid = sx * sx * ip0x * ip1y + sy * sy * ip1x * ip0y + EPS12;
                double p = (xin * sy * ip1x * ip0y - yin * sx * ip0x * ip1y) / mid;
                val = 0.5 * p + 0.5 * p;
            }
            qz[y + (long)x * (ny + 1)] = val;
        }
    free(ipbx); free(ipby); free(ippx); free(ippy);
    return 0;
}

/* Off-diagonal entry (0, 1) of the Gram matrix of the synthesis basis (row 3 of the reference's
   inner-product table at index 0, cuGetInnerProduct.cu:11-77, 92-126): the inner product of the
   synthesis functions of coefficients 0 and 1. */
static double ip_gram01(int dim, int wavelet, char bc) {
    int levels = 0;
    while ((2 << levels) <= dim) ++levels;
    double* e0 = (double*)calloc((size_t)dim, sizeof(double));
    double* e1 = (double*)calloc((size_t)dim, sizeof(double));
    e0[0] = 1.0;
    e1[1] = 1.0;
    or_dwt_line(e0, dim, levels, wavelet, bc, 0);
    or_dwt_line(e1, dim, levels, wavelet, bc, 0);
    double s = 0.0;
    for (int j = 0; j < dim; ++j) s += e0[j] * e1[j];
    free(e0);
    free(e1);
    return s;
}

/* GetDivL0Matrix (DivL0Matrix.cpp:3-46): the 4 x 4 map of the corner potentials of a 2D
   Dirichlet-wall projection, chosen by the difference of the two axes' levels.  The reference's entry
   for a difference of 5 is written with minus signs where the others have commas, so its first value
   is the sum of the four numbers and the other three are 0; it is evaluated here the same way. */
static void div_l0_matrix(double* dst, int lx, int ly) {
    int m = lx < ly ? lx : ly;
    int mx = lx - m, my = ly - m, k = mx > my ? mx : my;
    double r[4] = {-0.374999999999990, -0.124999999999991, -0.375000000000009, -0.125000000000009};
    static const double T[8][4] = {
        {-0.600000000000000, -0.400000000000000, -0.450000000000000, -0.050000000000000},
        {-1.058823529411764, -0.941176470588235, -0.485294117647059, -0.014705882352941},
        {-2.030769230769231, -1.969230769230771, -0.496153846153847, -0.003846153846153},
        {-4.015564202334636, -3.984435797665360, -0.499027237354084, -0.000972762645915},
        {0, 0, 0, 0},
        {-16.003905296558496, -15.996094703441514, -0.499938979741274, -0.000061020258726},
        {-32.001953005797915, -31.998046994202070, -0.499984742142203, -0.000015257857796},
        {-64.000976547601056, -63.999023452398980, -0.499996185360941, -0.000003814639067}};
    if (k == 5) {
        r[0] = -8.007804878048813 - 7.992195121951190 - 0.499756097560973 - 0.000243902439025;
        r[1] = r[2] = r[3] = 0.0;
    } else if (k >= 1 && k <= 8) {
        for (int i = 0; i < 4; ++i) r[i] = T[k - 1][i];
    }
    if (mx < my) {
        double t = r[0]; r[0] = r[2]; r[2] = t;
        t = r[1]; r[1] = r[3]; r[3] = t;
    }
    const double v[16] = {r[0], r[1], r[2], r[3], -r[0], -r[1], r[3], r[2],
                          r[1], r[0], -r[2], -r[3], -r[1], -r[0], -r[3], -r[2]};
    memcpy(dst, v, sizeof(v));
}

/* 2D local projection with Dirichlet domain walls (the recovery's bc 'd': base wavelet CDF4.6 with
   bc 'n', projection wavelet CDF3.7 with bc 'd'), cuProjectLocal_q_single_n
   (cuDivLocalProject.cu:1047-1460), launched by ProjectSingle (:2162-2198).  Entry (x, y) of qz, in
   [0, nx] x [0, ny], reads X(x, y) = xv(x, y - 1) and Y(x, y) = yv(x - 1, y) (0 outside):
   - x, y >= 2: the pointwise ratio P of the bc 'n' kernel (both passes, half each);
   - x in {0, 1}, y >= 2: the 2 x 2 solve of the pass along y, which couples the two wall-side
     coefficients X(0, y), X(1, y) with Y(1, y) through the base table's entries (0, 0) and (0, 1)
     at the scale dx_inv / nx;
   - y in {0, 1}, x >= 2: the same along x;
   - x, y in {0, 1}: the corner map (div_l0_matrix) of X(0, 1), X(1, 1), Y(1, 0), Y(1, 1). */
int or_project2d_nq(double* qz, const double* xv, const double* yv, int nx, int ny, double dx, double dy) {
    int Lx = ilog2(nx), Ly = ilog2(ny);
    if ((1 << Lx) != nx || (1 << Ly) != ny) return 1;
    double* pbx = (double*)malloc(sizeof(double) * (nx + 1));
    double* pby = (double*)malloc(sizeof(double) * (ny + 1));
    double* ppx = (double*)malloc(sizeof(double) * nx);
    double* ppy = (double*)malloc(sizeof(double) * ny);
    or_ip_diag(pbx, nx + 1, OR_CDF4_6, 'n');
    or_ip_diag(pby, ny + 1, OR_CDF4_6, 'n');
    or_ip_diag(ppx, nx, OR_CDF3_7, 'd');
    or_ip_diag(ppy, ny, OR_CDF3_7, 'd');
    const double gx = ip_gram01(nx + 1, OR_CDF4_6, 'n'), gy = ip_gram01(ny + 1, OR_CDF4_6, 'n');
    double l0[16];
    div_l0_matrix(l0, Lx, Ly);
    const double dxi = 1.0 / dx, dyi = 1.0 / dy;
#define XV(X_, Y_) ((Y_) > 0 ? xv[((Y_) - 1) + (long)(X_) * ny] : 0.0)
#define YV(X_, Y_) ((X_) > 0 ? yv[(Y_) + (long)((X_) - 1) * (ny + 1)] : 0.0)
    for (int x = 0; x <= nx; ++x)
        for (int y = 0; y <= ny; ++y) {
            const double sx = 4.0 * dxi / ((double)(1 << (Lx - bitlen(x > 0 ? x - 1 : 0) + 1)) + EPS12);
            const double sy = 4.0 * dyi / ((double)(1 << (Ly - bitlen(y > 0 ? y - 1 : 0) + 1)) + EPS12);
            double qy = 0.0, qx = 0.0;
            if (x >= 2 && y >= 2) {
                const double ip0x = ppx[x - 1], ip1x = pbx[x], ip0y = ppy[y - 1], ip1y = pby[y];
                const double X = XV(x, y), Y = YV(x, y);
                const double m1 = sx * sx * ip0x * ip1y + sy * sy * ip1x * ip0y + EPS12;
                qy = 0.5 * ((X * sy * ip1x * ip0y - Y * sx * ip0x * ip1y) / m1);
                const double m2 = sy * sy * ip0y * ip1x + sx * sx * ip1y * ip0x + EPS12;
                qx = 0.5 * ((X * sy * ip0y * ip1x - Y * sx * ip1y * ip0x) / m2);
            } else if (y >= 2) {  /* x in {0, 1}: the pass along y */
                const double se = dxi / nx, ip0x = ppx[0], b00 = pbx[0], b01 = gx;
                const double ip0y = ppy[y - 1], ip1y = pby[y];
                const double ye = YV(1, y), x0 = XV(0, y), x1 = XV(1, y);
                double m0 = se * se * ip0x * ip1y + sy * sy * b00 * ip0y;
                double m1 = -se * se * ip0x * ip1y + sy * sy * b01 * ip0y;
                const double dv = m0 * m0 - m1 * m1 + EPS12;
                m0 /= dv;
                m1 /= -dv;
                double f1 = ye * se * ip0x * ip1y;
                f1 += x0 * sy * b00 * ip0y;
                f1 += x1 * sy * b01 * ip0y;
                double f2 = -ye * se * ip0x * ip1y;
                f2 += x0 * sy * b01 * ip0y;
                f2 += x1 * sy * b00 * ip0y;
                qy = x == 0 ? m0 * f1 + m1 * f2 : m1 * f1 + m0 * f2;
            } else if (x >= 2) {  /* y in {0, 1}: the pass along x */
                const double se = dyi / ny, ip0y = ppy[0], b00 = pby[0], b01 = gy;
                const double ip0x = ppx[x - 1], ip1x = pbx[x];
                const double xe = XV(x, 1), y0 = YV(x, 0), y1 = YV(x, 1);
                double m0 = sx * sx * ip0x * b00 + se * se * ip1x * ip0y;
                double m1 = sx * sx * ip0x * b01 - se * se * ip1x * ip0y;
                const double dv = m0 * m0 - m1 * m1 + EPS12;
                m0 /= dv;
                m1 /= -dv;
                const double a00 = ip0x * b00, a01 = ip0x * b01;
                double f1 = -xe * se * ip1x * ip0y;
                f1 -= y0 * sx * a00;
                f1 -= y1 * sx * a01;
                double f2 = xe * se * ip1x * ip0y;
                f2 -= y0 * sx * a01;
                f2 -= y1 * sx * a00;
                qx = y == 0 ? m0 * f1 + m1 * f2 : m1 * f1 + m0 * f2;
            } else {  /* the corner */
                const double* a = l0 + 4 * (2 * y + x);
                qx = a[2] * XV(0, 1) + a[3] * XV(1, 1) - a[0] * YV(1, 0) - a[1] * YV(1, 1);
            }
            qz[y + (long)x * (ny + 1)] = qx + qy;
        }
#undef XV
#undef YV
    free(pbx); free(pby); free(ppx); free(ppy);
    return 0;
}

/* ----------------------------------------------------------- potential recovery ---- */
/* CuWaveletPotentialRecover3D::Solve (cuWaveletPotentialRecover3D.cu:16-61) */
int or_recover3d(double* qx, double* qy, double* qz, const double* xv, const double* yv, const double* zv,
                 int nx, int ny, int nz, double dx, double dy, double dz, char bc) {
    /* bc: the walls' boundary type (cuWaveletPotentialRecover3D.cu:6-11); the div wavelet takes the
       other one (proj_bc) and the projection kernel follows it */
    if (bc != 'n' && bc != 'd') return 2;
    int Lx = ilog2(nx), Ly = ilog2(ny), Lz = ilog2(nz);
    char bcd = bc == 'n' ? 'd' : 'n';
    size_t sxv = (size_t)(nx + 1) * ny * nz, syv = (size_t)nx * (ny + 1) * nz, szv = (size_t)nx * ny * (nz + 1);
    double* tx = (double*)malloc(sizeof(double) * sxv);
    double* ty = (double*)malloc(sizeof(double) * syv);
    double* tz = (double*)malloc(sizeof(double) * szv);
    memcpy(tx, xv, sizeof(double) * sxv);
    memcpy(ty, yv, sizeof(double) * syv);
    memcpy(tz, zv, sizeof(double) * szv);
    int e = 0;
    e |= or_dwt_axis(tx, nx + 1, ny, nz, Lx, 'x', OR_CDF4_6, bcd, 1);
    e |= or_dwt_axis(tx, nx + 1, ny, nz, Ly, 'y', OR_CDF3_7, bc, 1);
    e |= or_dwt_axis(tx, nx + 1, ny, nz, Lz, 'z', OR_CDF3_7, bc, 1);
    e |= or_dwt_axis(ty, nx, ny + 1, nz, Lx, 'x', OR_CDF3_7, bc, 1);
    e |= or_dwt_axis(ty, nx, ny + 1, nz, Ly, 'y', OR_CDF4_6, bcd, 1);
    e |= or_dwt_axis(ty, nx, ny + 1, nz, Lz, 'z', OR_CDF3_7, bc, 1);
    e |= or_dwt_axis(tz, nx, ny, nz + 1, Lx, 'x', OR_CDF3_7, bc, 1);
    e |= or_dwt_axis(tz, nx, ny, nz + 1, Ly, 'y', OR_CDF3_7, bc, 1);
    e |= or_dwt_axis(tz, nx, ny, nz + 1, Lz, 'z', OR_CDF4_6, bcd, 1);
    e |= bc == 'n' ? or_project3d(qx, qy, qz, tx, ty, tz, nx, ny, nz, dx, dy, dz)
                   : or_project3d_nq(qx, qy, qz, tx, ty, tz, nx, ny, nz, dx, dy, dz);
    e |= or_dwt_axis(qx, nx, ny + 1, nz + 1, Lx, 'x', OR_CDF3_7, bc, 0);
    e |= or_dwt_axis(qx, nx, ny + 1, nz + 1, Ly, 'y', OR_CDF4_6, bcd, 0);
    e |= or_dwt_axis(qx, nx, ny + 1, nz + 1, Lz, 'z', OR_CDF4_6, bcd, 0);
    e |= or_dwt_axis(qy, nx + 1, ny, nz + 1, Lx, 'x', OR_CDF4_6, bcd, 0);
    e |= or_dwt_axis(qy, nx + 1, ny, nz + 1, Ly, 'y', OR_CDF3_7, bc, 0);
    e |= or_dwt_axis(qy, nx + 1, ny, nz + 1, Lz, 'z', OR_CDF4_6, bcd, 0);
    e |= or_dwt_axis(qz, nx + 1, ny + 1, nz, Lx, 'x', OR_CDF4_6, bcd, 0);
    e |= or_dwt_axis(qz, nx + 1, ny + 1, nz, Ly, 'y', OR_CDF4_6, bcd, 0);
    e |= or_dwt_axis(qz, nx + 1, ny + 1, nz, Lz, 'z', OR_CDF3_7, bc, 0);
    free(tx); free(ty); free(tz);
    return e;
}

/* CuWaveletPotentialRecover3D::CutCoefficients (cuWaveletPotentialRecover3D.cu:123-239), in place:
   analysis with the recovery's synthesis wavelets, cuCutCoefs over the (nx+1, ny+1, nz+1) index box
   (coefficient level j = L - bitlength(max(i - 1, 0)) per axis; a cell with some j below `level`
   clears qx at (x-1, y, z), qy at (x, y-1, z), qz at (x, y, z-1) with the reference's guards), then
   synthesis.  Returns 1 for a level outside [0, min L]. */
int or_cut3d(double* qx, double* qy, double* qz, int nx, int ny, int nz, int level) {
    int Lx = ilog2(nx), Ly = ilog2(ny), Lz = ilog2(nz);
    int Lmin = Lx < Ly ? (Lx < Lz ? Lx : Lz) : (Ly < Lz ? Ly : Lz);
    if (level < 0 || level > Lmin) return 1;
    char bc = 'n', bcd = 'd';
    int e = 0;
    e |= or_dwt_axis(qx, nx, ny + 1, nz + 1, Lx, 'x', OR_CDF3_7, bc, 1);
    e |= or_dwt_axis(qx, nx, ny + 1, nz + 1, Ly, 'y', OR_CDF4_6, bcd, 1);
    e |= or_dwt_axis(qx, nx, ny + 1, nz + 1, Lz, 'z', OR_CDF4_6, bcd, 1);
    e |= or_dwt_axis(qy, nx + 1, ny, nz + 1, Lx, 'x', OR_CDF4_6, bcd, 1);
    e |= or_dwt_axis(qy, nx + 1, ny, nz + 1, Ly, 'y', OR_CDF3_7, bc, 1);
    e |= or_dwt_axis(qy, nx + 1, ny, nz + 1, Lz, 'z', OR_CDF4_6, bcd, 1);
    e |= or_dwt_axis(qz, nx + 1, ny + 1, nz, Lx, 'x', OR_CDF4_6, bcd, 1);
    e |= or_dwt_axis(qz, nx + 1, ny + 1, nz, Ly, 'y', OR_CDF4_6, bcd, 1);
    e |= or_dwt_axis(qz, nx + 1, ny + 1, nz, Lz, 'z', OR_CDF3_7, bc, 1);
    for (int z = 0; z <= nz; ++z)
        for (int x = 0; x <= nx; ++x)
            for (int y = 0; y <= ny; ++y) {
                int jx = Lx - bitlen(x - 1 > 0 ? x - 1 : 0);
                int jy = Ly - bitlen(y - 1 > 0 ? y - 1 : 0);
                int jz = Lz - bitlen(z - 1 > 0 ? z - 1 : 0);
                long iqx = y + (long)(x - 1) * (ny + 1) + (long)z * nx * (ny + 1);
                long iqy = (y - 1) + (long)x * ny + (long)z * (nx + 1) * ny;
                long iqz = y + (long)x * (ny + 1) + (long)(z - 1) * (nx + 1) * (ny + 1);
                if (jx < level) {
                    qx[iqx] = 0.0;
                    if (y > 0) qy[iqy] = 0.0;
                    if (z > 0) qz[iqz] = 0.0;
                }
                if (jy < level) {
                    qy[iqy] = 0.0;
                    if (x > 0) qx[iqx] = 0.0;
                    if (z > 0) qz[iqz] = 0.0;
                }
                if (jz < level) {
                    qz[iqz] = 0.0;
                    if (x > 0) qx[iqx] = 0.0;
                    if (y > 0) qy[iqy] = 0.0;
                }
            }
    e |= or_dwt_axis(qx, nx, ny + 1, nz + 1, Lx, 'x', OR_CDF3_7, bc, 0);
    e |= or_dwt_axis(qx, nx, ny + 1, nz + 1, Ly, 'y', OR_CDF4_6, bcd, 0);
    e |= or_dwt_axis(qx, nx, ny + 1, nz + 1, Lz, 'z', OR_CDF4_6, bcd, 0);
    e |= or_dwt_axis(qy, nx + 1, ny, nz + 1, Lx, 'x', OR_CDF4_6, bcd, 0);
    e |= or_dwt_axis(qy, nx + 1, ny, nz + 1, Ly, 'y', OR_CDF3_7, bc, 0);
    e |= or_dwt_axis(qy, nx + 1, ny, nz + 1, Lz, 'z', OR_CDF4_6, bcd, 0);
    e |= or_dwt_axis(qz, nx + 1, ny + 1, nz, Lx, 'x', OR_CDF4_6, bcd, 0);
    e |= or_dwt_axis(qz, nx + 1, ny + 1, nz, Ly, 'y', OR_CDF4_6, bcd, 0);
    e |= or_dwt_axis(qz, nx + 1, ny + 1, nz, Lz, 'z', OR_CDF3_7, bc, 0);
    return e;
}

/* CuWaveletPotentialRecover2D::Solve (cuWaveletPotentialRecover2D.cu:16-36) */
int or_recover2d(double* qz, const double* xv, const double* yv, int nx, int ny, double dx, double dy, char bc) {
    if (bc != 'n' && bc != 'd') return 2;
    const char bcd = bc == 'n' ? 'd' : 'n';
    int Lx = ilog2(nx), Ly = ilog2(ny);
    size_t sxv = (size_t)(nx + 1) * ny, syv = (size_t)nx * (ny + 1);
    double* tx = (double*)malloc(sizeof(double) * sxv);
    double* ty = (double*)malloc(sizeof(double) * syv);
    memcpy(tx, xv, sizeof(double) * sxv);
    memcpy(ty, yv, sizeof(double) * syv);
    int e = 0;
    e |= or_dwt_axis(tx, nx + 1, ny, 1, Lx, 'x', OR_CDF4_6, bcd, 1);
    e |= or_dwt_axis(tx, nx + 1, ny, 1, Ly, 'y', OR_CDF3_7, bc, 1);
    e |= or_dwt_axis(ty, nx, ny + 1, 1, Lx, 'x', OR_CDF3_7, bc, 1);
    e |= or_dwt_axis(ty, nx, ny + 1, 1, Ly, 'y', OR_CDF4_6, bcd, 1);
    e |= bc == 'n' ? or_project2d(qz, tx, ty, nx, ny, dx, dy) : or_project2d_nq(qz, tx, ty, nx, ny, dx, dy);
    e |= or_dwt_axis(qz, nx + 1, ny + 1, 1, Lx, 'x', OR_CDF4_6, bcd, 0);
    e |= or_dwt_axis(qz, nx + 1, ny + 1, 1, Ly, 'y', OR_CDF4_6, bcd, 0);
    free(tx); free(ty);
    return e;
}

/* ------------------------------------------------------------------------- curl ---- */
void or_curl3d(double* xv, double* yv, double* zv, const double* qx, const double* qy, const double* qz,
               int nx, int ny, int nz, double dx, double dy, double dz) {
    double dxi = 1.0 / dx, dyi = 1.0 / dy, dzi = 1.0 / dz;
    long sqx = (long)nx * (ny + 1), sqy = (long)(nx + 1) * ny, sqz = (long)(nx + 1) * (ny + 1);
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int x = 0; x <= nx; ++x)
            for (int y = 0; y < ny; ++y) {
                long iqz = y + (long)x * (ny + 1) + z * sqz, iqy = y + (long)x * ny + z * sqy;
                xv[y + (long)x * ny + (long)z * (nx + 1) * ny] =
                    (qz[iqz + 1] - qz[iqz]) * dyi - (qy[iqy + sqy] - qy[iqy]) * dzi;
            }
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y <= ny; ++y) {
                long iqz = y + (long)x * (ny + 1) + z * sqz, iqx = y + (long)x * (ny + 1) + z * sqx;
                yv[y + (long)x * (ny + 1) + (long)z * nx * (ny + 1)] =
                    (qx[iqx + sqx] - qx[iqx]) * dzi - (qz[iqz + (ny + 1)] - qz[iqz]) * dxi;
            }
#pragma omp parallel for schedule(static)
    for (int z = 0; z <= nz; ++z)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y) {
                long iqx = y + (long)x * (ny + 1) + z * sqx, iqy = y + (long)x * ny + z * sqy;
                zv[y + (long)x * ny + (long)z * nx * ny] = (qy[iqy + ny] - qy[iqy]) * dxi - (qx[iqx + 1] - qx[iqx]) * dyi;
            }
}

void or_curl2d(double* xv, double* yv, const double* qz, int nx, int ny, double dx, double dy) {
    for (int x = 0; x <= nx; ++x)
        for (int y = 0; y < ny; ++y) {
            long iq = y + (long)x * (ny + 1);
            xv[y + (long)x * ny] = (qz[iq + 1] - qz[iq]) / dy;
        }
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y <= ny; ++y) {
            long iq = y + (long)x * (ny + 1);
            yv[y + (long)x * (ny + 1)] = -(qz[iq + ny + 1] - qz[iq]) / dx;
        }
}

/* ---------------------------------------------------------- divergence / gradient ---- */
void or_divergence3d(double* b, const double* xv, const double* yv, const double* zv,
                     const double* ax, const double* ay, const double* az, int nx, int ny, int nz,
                     double dx, double dy, double dz) {
    double dxi = 1.0 / dx, dyi = 1.0 / dy, dzi = 1.0 / dz;
    long sxv = (long)(nx + 1) * ny, syv = (long)nx * (ny + 1), szv = (long)nx * ny;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y) {
                long ix = y + (long)x * ny + z * sxv, iy = y + (long)x * (ny + 1) + z * syv, iz = y + (long)x * ny + z * szv;
                double v = (xv[ix + ny] * ax[ix + ny] - xv[ix] * ax[ix]) * dxi +
                           (yv[iy + 1] * ay[iy + 1] - yv[iy] * ay[iy]) * dyi +
                           (zv[iz + szv] * az[iz + szv] - zv[iz] * az[iz]) * dzi;
                b[y + (long)x * ny + z * szv] = -v;
            }
}

void or_divergence2d(double* b, const double* xv, const double* yv, const double* ax, const double* ay,
                     int nx, int ny, double dx, double dy) {
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y) {
            long ix = y + (long)x * ny, iy = y + (long)x * (ny + 1);
            double v = (xv[ix + ny] * ax[ix + ny] - xv[ix] * ax[ix]) / dx + (yv[iy + 1] * ay[iy + 1] - yv[iy] * ay[iy]) / dy;
            b[ix] = -v;
        }
}

void or_grad_subtract3d(double* xv, double* yv, double* zv, const double* p,
                        const double* ax, const double* ay, const double* az, int nx, int ny, int nz,
                        double dx, double dy, double dz, int multiply_frac) {
    long sxv = (long)(nx + 1) * ny, syv = (long)nx * (ny + 1), sp = (long)nx * ny;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z) {
        for (int x = 0; x <= nx; ++x)
            for (int y = 0; y < ny; ++y) {
                long i = y + (long)x * ny + z * sxv;
                double g = 0.0;
                if (x > 0 && x < nx && ax[i] > EPS12) {
                    long ip = y + (long)x * ny + z * sp;
                    g = (p[ip] - p[ip - ny]) / (dx + dx) * 2.0;
                }
                xv[i] -= g;
                if (multiply_frac) xv[i] *= ax[i];
            }
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y <= ny; ++y) {
                long i = y + (long)x * (ny + 1) + z * syv;
                double g = 0.0;
                if (y > 0 && y < ny && ay[i] > EPS12) {
                    long ip = y + (long)x * ny + z * sp;
                    g = (p[ip] - p[ip - 1]) / (dy + dy) * 2.0;
                }
                yv[i] -= g;
                if (multiply_frac) yv[i] *= ay[i];
            }
    }
#pragma omp parallel for schedule(static)
    for (int z = 0; z <= nz; ++z)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y) {
                long i = y + (long)x * ny + z * sp;
                double g = 0.0;
                if (z > 0 && z < nz && az[i] > EPS12) g = (p[i] - p[i - sp]) / (dz + dz) * 2.0;
                zv[i] -= g;
                if (multiply_frac) zv[i] *= az[i];
            }
}

void or_grad_subtract2d(double* xv, double* yv, const double* p, const double* ax, const double* ay,
                        int nx, int ny, double dx, double dy, int multiply_frac) {
    for (int x = 0; x <= nx; ++x)
        for (int y = 0; y < ny; ++y) {
            long i = y + (long)x * ny;
            double g = 0.0;
            if (x > 0 && x < nx && ax[i] > EPS12) g = (p[i] - p[i - ny]) / (dx + dx) * 2.0;
            xv[i] -= g;
            if (multiply_frac) xv[i] *= ax[i];
        }
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y <= ny; ++y) {
            long i = y + (long)x * (ny + 1);
            double g = 0.0;
            if (y > 0 && y < ny && ay[i] > EPS12) {
                long ip = y + (long)x * ny;
                g = (p[ip] - p[ip - 1]) / (dy + dy) * 2.0;
            }
            yv[i] -= g;
            if (multiply_frac) yv[i] *= ay[i];
        }
}

/* --------------------------------------------------------------- solids ---- */
/* cuInitLsSphere (cuSolidLevelSet3D.cu:11-27), extended to a union (min) of spheres */
void or_sdf_spheres3d(double* sdf, int nx, int ny, int nz, double dx, const double* centers, const double* radii,
                      int nspheres) {
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y) {
                double px = (x + 0.5) * dx, py = (y + 0.5) * dx, pz = (z + 0.5) * dx;
                double best = 1e300;
                for (int s = 0; s < nspheres; ++s) {
                    double ddx = px - centers[3 * s], ddy = py - centers[3 * s + 1], ddz = pz - centers[3 * s + 2];
                    double d = sqrt(ddx * ddx + ddy * ddy + ddz * ddz) - radii[s];
                    if (d < best) best = d;
                }
                sdf[y + (long)x * ny + (long)z * nx * ny] = best;
            }
}

/* union with axis-aligned boxes: exact box signed distance, combined by min */
void or_sdf_boxes3d(double* sdf, int nx, int ny, int nz, double dx, const double* lo, const double* hi, int nboxes) {
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y) {
                double p[3] = {(x + 0.5) * dx, (y + 0.5) * dx, (z + 0.5) * dx};
                long i = y + (long)x * ny + (long)z * nx * ny;
                double best = sdf[i];
                for (int b = 0; b < nboxes; ++b) {
                    double q[3], out = 0.0, inside = -1e300;
                    for (int c = 0; c < 3; ++c) {
                        double ctr = 0.5 * (lo[3 * b + c] + hi[3 * b + c]), half = 0.5 * (hi[3 * b + c] - lo[3 * b + c]);
                        q[c] = fabs(p[c] - ctr) - half;
                        if (q[c] > 0) out += q[c] * q[c];
                        if (q[c] > inside) inside = q[c];
                    }
                    double d = sqrt(out) + (inside < 0 ? inside : 0.0);
                    if (d < best) best = d;
                }
                sdf[i] = best;
            }
}

/* cuComputeFrac (cuSolidLevelSet3D.cu:29-35) */
static double frac_from_ls(double dx, double l, double r) {
    double dif = r - l;
    double q = dx * dx - dif * dif;
    double d = sqrt(q > 1e-14 ? q : 1e-14);
    double t = (1.0 - (r + l) / d) * 0.5;
    if (t < 0.0) t = 0.0;
    if (t > 1.0) t = 1.0;
    return 1.0 - t;
}

/* cuGetAx/Ay/Az (cuSolidLevelSet3D.cu:36-90): boundary faces use the adjacent cell twice */
void or_fractions3d(double* ax, double* ay, double* az, const double* sdf, int nx, int ny, int nz, double dx) {
    long s = (long)nx * ny;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z) {
        for (int x = 0; x <= nx; ++x)
            for (int y = 0; y < ny; ++y) {
                int xl = x - 1 < 0 ? 0 : x - 1, xr = x < nx - 1 ? x : nx - 1;
                ax[y + (long)x * ny + (long)z * (nx + 1) * ny] =
                    frac_from_ls(dx, sdf[y + (long)xl * ny + z * s], sdf[y + (long)xr * ny + z * s]);
            }
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y <= ny; ++y) {
                int yl = y - 1 < 0 ? 0 : y - 1, yr = y < ny - 1 ? y : ny - 1;
                ay[y + (long)x * (ny + 1) + (long)z * nx * (ny + 1)] =
                    frac_from_ls(dx, sdf[yl + (long)x * ny + z * s], sdf[yr + (long)x * ny + z * s]);
            }
    }
#pragma omp parallel for schedule(static)
    for (int z = 0; z <= nz; ++z)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y) {
                int zl = z - 1 < 0 ? 0 : z - 1, zr = z < nz - 1 ? z : nz - 1;
                az[y + (long)x * ny + (long)z * s] = frac_from_ls(dx, sdf[y + (long)x * ny + zl * s], sdf[y + (long)x * ny + zr * s]);
            }
}

void or_fractions2d(double* ax, double* ay, const double* sdf, int nx, int ny, double dx) {
    for (int x = 0; x <= nx; ++x)
        for (int y = 0; y < ny; ++y) {
            int xl = x - 1 < 0 ? 0 : x - 1, xr = x < nx - 1 ? x : nx - 1;
            ax[y + (long)x * ny] = frac_from_ls(dx, sdf[y + (long)xl * ny], sdf[y + (long)xr * ny]);
        }
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y <= ny; ++y) {
            int yl = y - 1 < 0 ? 0 : y - 1, yr = y < ny - 1 ? y : ny - 1;
            ay[y + (long)x * (ny + 1)] = frac_from_ls(dx, sdf[yl + (long)x * ny], sdf[yr + (long)x * ny]);
        }
}

/* --------------------------------------------- subsampled face fractions of a level set ---- */
/* CuSolidLevelSet3D::GetFrac(ax, ay, az, ls, dim, dx) (cuSolidLevelSet3D.cu:356-372) with
   cuGetAx/Ay/Az_divide (:164-316); InterpolateQuadratic3D (Interpolation.cuh:119-156),
   InterpolateLinear3D with cuGetIxFx (:16-29, 80-117), CLAMP_L of the double build (:9) */
static const double OR_CLAMP_L = (double)1e-10f;

static double ls_quadratic3(const double* ls, double x, double y, double z, int nx, int ny, int nz) {
    int ix = (int)floor(x - 0.5), iy = (int)floor(y - 0.5), iz = (int)floor(z - 0.5);
    double fx = x - ix, fy = y - iy, fz = z - iz;
    double wx[3] = {0.5 * (1.5 - fx) * (1.5 - fx), 0.75 - (fx - 1.0) * (fx - 1.0), 0.5 * (fx - 0.5) * (fx - 0.5)};
    double wy[3] = {0.5 * (1.5 - fy) * (1.5 - fy), 0.75 - (fy - 1.0) * (fy - 1.0), 0.5 * (fy - 0.5) * (fy - 0.5)};
    double wz[3] = {0.5 * (1.5 - fz) * (1.5 - fz), 0.75 - (fz - 1.0) * (fz - 1.0), 0.5 * (fz - 0.5) * (fz - 0.5)};
    double r = 0.0;
    for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                int xx = ix + j < 0 ? 0 : (ix + j > nx - 1 ? nx - 1 : ix + j);
                int yy = iy + i < 0 ? 0 : (iy + i > ny - 1 ? ny - 1 : iy + i);
                int zz = iz + k < 0 ? 0 : (iz + k > nz - 1 ? nz - 1 : iz + k);
                r += wx[j] * wy[i] * wz[k] * ls[yy + (long)xx * ny + (long)zz * nx * ny];
            }
    return r;
}

static void ixfx(int* i, double* f, double x, int n) {
    if (x < OR_CLAMP_L) x = OR_CLAMP_L;
    *i = (int)x;
    if (*i >= n - 1) { *i = n - 2; *f = 1.0; } /* 1.f - CLAMP_L is 1 in float */
    else *f = x - *i;
}

static double ls_linear3(const double* ls, double x, double y, double z, int nx, int ny, int nz) {
    int ix, iy, iz;
    double fx, fy, fz;
    ixfx(&ix, &fx, x, nx);
    ixfx(&iy, &fy, y, ny);
    ixfx(&iz, &fz, z, nz);
    double wx0 = 1 - fx, wy0 = 1 - fy, wz0 = 1 - fz;
    long sl = (long)nx * ny, i0 = iy + (long)ix * ny + iz * sl;
    double r = ls[i0] * wx0 * wy0 * wz0;
    r += ls[i0 + 1] * wx0 * fy * wz0;
    r += ls[i0 + ny] * fx * wy0 * wz0;
    r += ls[i0 + ny + 1] * fx * fy * wz0;
    i0 += sl;
    r += ls[i0] * wx0 * wy0 * fz;
    r += ls[i0 + 1] * wx0 * fy * fz;
    r += ls[i0 + ny] * fx * wy0 * fz;
    r += ls[i0 + ny + 1] * fx * fy * fz;
    return r;
}

void or_fractions3d_subsampled(double* ax, double* ay, double* az, const double* ls, int nx, int ny, int nz, double dx) {
    double inv = 1.0 / dx, dsub = dx / 128, half = 0.5 * dsub;
    for (int a = 0; a < 3; ++a) {
        int ex = nx + (a == 0), ey = ny + (a == 1), ez = nz + (a == 2);
        double* out = a == 0 ? ax : (a == 1 ? ay : az);
#pragma omp parallel for schedule(dynamic, 4)
        for (int z = 0; z < ez; ++z)
            for (int x = 0; x < ex; ++x)
                for (int y = 0; y < ey; ++y) {
                    double px = (a == 0 ? (double)x : x + 0.5) * dx, py = (a == 1 ? (double)y : y + 0.5) * dx;
                    double pz = (a == 2 ? (double)z : z + 0.5) * dx;
                    double v = ls_quadratic3(ls, px * inv - 0.5, py * inv - 0.5, pz * inv - 0.5, nx, ny, nz);
                    double res = 0.0;
                    if (v > dx) {
                        res = 1.0;
                    } else if (v > -dx) {
                        int cnt = 0;
                        for (int o = 0; o < 128; ++o)
                            for (int in = 0; in < 128; ++in) {
                                double qx, qy, qz;
                                if (a == 0) { qx = x * dx; qy = y * dx + half + in * dsub; qz = z * dx + half + o * dsub; }
                                else if (a == 1) { qx = x * dx + half + in * dsub; qy = y * dx; qz = z * dx + half + o * dsub; }
                                else { qx = x * dx + half + o * dsub; qy = y * dx + half + in * dsub; qz = z * dx; }
                                if (ls_linear3(ls, qx * inv - 0.5, qy * inv - 0.5, qz * inv - 0.5, nx, ny, nz) > 0.0) ++cnt;
                            }
                        res = cnt * (1.0 / 16384.0);
                    }
                    out[y + (long)x * ey + (long)z * ex * ey] = res < 0.0 ? 0.0 : (res > 1.0 ? 1.0 : res);
                }
    }
}

/* -------------------------------------------------------------- fast sweeping ---- */
/* CuFastSweeping::Solve / ReinitLevelSet (cuFastSweeping.cu:98-140, 215-257, 383-396): Jacobi
   iterations (each reads the previous iterate) of the upwind eikonal update on cells above -1e-12 */
static double eikonal3(double mx, double my, double mz, double h) {
    double m[3] = {mx, my, mz};
    for (int i = 1; i < 3; ++i)
        for (int j = 0; j < 3 - i; ++j)
            if (m[j] > m[j + 1]) { double t = m[j]; m[j] = m[j + 1]; m[j + 1] = t; }
    double d2 = h * h, r = m[0] + h;
    if (r > m[1]) {
        double s = sqrt(-m[0] * m[0] + 2 * m[0] * m[1] - m[1] * m[1] + 2 * d2);
        r = (m[1] * d2 + m[0] * d2 + d2 * s) / (2 * d2);
        if (r > m[2]) {
            double a = sqrt(d2 * (-2 * m[0] * m[0] - 2 * m[1] * m[1] - 2 * m[2] * m[2] + 2 * m[0] * m[1] +
                                  2 * m[0] * m[2] + 2 * m[1] * m[2]) + 3 * d2 * d2);
            r = (d2 * d2 * (m[0] + m[1] + m[2]) + h * d2 * a) / (3 * d2 * d2);
        }
    }
    return r;
}

static void fsweep3(double* ls, int nx, int ny, int nz, double h, int iters) {
    long n = (long)nx * ny * nz, sl = (long)nx * ny;
    double* prev = (double*)malloc(sizeof(double) * n);
    for (int it = 0; it < iters; ++it) {
        memcpy(prev, ls, sizeof(double) * n);
#pragma omp parallel for schedule(static)
        for (int z = 0; z < nz; ++z)
            for (int x = 0; x < nx; ++x)
                for (int y = 0; y < ny; ++y) {
                    long i = y + (long)x * ny + z * sl;
                    if (!(prev[i] > -1e-12)) continue;
                    double big = 1e8;
                    double l = x > 0 ? prev[i - ny] : big, r = x < nx - 1 ? prev[i + ny] : big;
                    double u = y < ny - 1 ? prev[i + 1] : big, d = y > 0 ? prev[i - 1] : big;
                    double f = z > 0 ? prev[i - sl] : big, b = z < nz - 1 ? prev[i + sl] : big;
                    ls[i] = eikonal3(l < r ? l : r, u < d ? u : d, f < b ? f : b, h);
                }
    }
    free(prev);
}

/* CuFastSweeping::ParticlesToLs (cuFastSweeping.cu:259-349); cells outside the grid are skipped */
void or_particles_to_ls(double* ls, const double* xyz, int count, int nx, int ny, int nz, double dx, double radius,
                        double max_dis, int iters) {
    long n = (long)nx * ny * nz;
    for (long i = 0; i < n; ++i) ls[i] = dx;
    for (int p = 0; p < count; ++p) {
        double x = xyz[3 * p] / dx - 0.5, y = xyz[3 * p + 1] / dx - 0.5, z = xyz[3 * p + 2] / dx - 0.5;
        int ix = (int)floor(x), iy = (int)floor(y), iz = (int)floor(z);
        double fx = x - ix, fy = y - iy, fz = z - iz;
        double wx[2] = {fx * fx, (1 - fx) * (1 - fx)}, wy[2] = {fy * fy, (1 - fy) * (1 - fy)};
        double wz[2] = {fz * fz, (1 - fz) * (1 - fz)};
        for (int k = 0; k < 2; ++k)
            for (int j = 0; j < 2; ++j)
                for (int i = 0; i < 2; ++i) {
                    int cx = ix + j, cy = iy + i, cz = iz + k;
                    if (cx < 0 || cx >= nx || cy < 0 || cy >= ny || cz < 0 || cz >= nz) continue;
                    double d = sqrt(wx[j] + wy[i] + wz[k]) * dx - radius;
                    long q = cy + (long)cx * ny + (long)cz * nx * ny;
                    if (d < ls[q]) ls[q] = d;
                }
    }
    for (int pass = 0; pass < 2; ++pass) {
        for (long i = 0; i < n; ++i) ls[i] = ls[i] > 0.0 ? -ls[i] : max_dis;
        fsweep3(ls, nx, ny, nz, dx, iters);
    }
    for (long i = 0; i < n; ++i) ls[i] = -ls[i];
}

/* CuFastSweeping::ParticlesToLsNarrow (cuFastSweeping.cu:352-385): ls is the caller's start (not
   filled); the particles lower it as above, then n_iters sweeps, negation, n_iters sweeps (max_dis
   is not used); cells outside the grid are skipped */
void or_particles_to_ls_narrow(double* ls, const double* xyz, int count, int nx, int ny, int nz, double dx,
                               double radius, int iters) {
    long n = (long)nx * ny * nz;
    for (int p = 0; p < count; ++p) {
        double x = xyz[3 * p] / dx - 0.5, y = xyz[3 * p + 1] / dx - 0.5, z = xyz[3 * p + 2] / dx - 0.5;
        int ix = (int)floor(x), iy = (int)floor(y), iz = (int)floor(z);
        double fx = x - ix, fy = y - iy, fz = z - iz;
        double wx[2] = {fx * fx, (1 - fx) * (1 - fx)}, wy[2] = {fy * fy, (1 - fy) * (1 - fy)};
        double wz[2] = {fz * fz, (1 - fz) * (1 - fz)};
        for (int k = 0; k < 2; ++k)
            for (int j = 0; j < 2; ++j)
                for (int i = 0; i < 2; ++i) {
                    int cx = ix + j, cy = iy + i, cz = iz + k;
                    if (cx < 0 || cx >= nx || cy < 0 || cy >= ny || cz < 0 || cz >= nz) continue;
                    double d = sqrt(wx[j] + wy[i] + wz[k]) * dx - radius;
                    long q = cy + (long)cx * ny + (long)cz * nx * ny;
                    if (d < ls[q]) ls[q] = d;
                }
    }
    fsweep3(ls, nx, ny, nz, dx, iters);
    for (long i = 0; i < n; ++i) ls[i] = -ls[i];
    fsweep3(ls, nx, ny, nz, dx, iters);
}

void or_fast_sweep(double* ls, int nx, int ny, int nz, double dx, int iters, int reinit) {
    long n = (long)nx * ny * nz;
    if (reinit) {
        for (long i = 0; i < n; ++i) ls[i] = -ls[i];
        fsweep3(ls, nx, ny, nz, dx, iters);
        for (long i = 0; i < n; ++i) ls[i] = -ls[i];
    }
    fsweep3(ls, nx, ny, nz, dx, iters);
}

/* ------------------------------------------------------- fractional multigrid 3D ---- */
/* cuWjFrac3D_n (cuWeightedJacobi3D.cu:620-695): Neumann walls, cut-cell face weights */
static inline void frac_row3d(const double* v, const double* ax, const double* ay, const double* az,
                              int nx, int ny, int nz, const double* dxs, const double* dys, const double* dzs,
                              int x, int y, int z, double* diag, double* off) {
    long i = y + (long)x * ny + (long)z * nx * ny, sl = (long)nx * ny;
    long iax = y + (long)x * ny + (long)z * (nx + 1) * ny, iay = y + (long)x * (ny + 1) + (long)z * nx * (ny + 1);
    double dg = 0.0, od = 0.0, cf;
    if (y > 0) { cf = ay[iay] / (dys[y - 1] + dys[y]) / dys[y] * 2.0; dg += cf; od += -cf * v[i - 1]; }
    if (y < ny - 1) { cf = ay[iay + 1] / (dys[y + 1] + dys[y]) / dys[y] * 2.0; dg += cf; od += -cf * v[i + 1]; }
    if (x > 0) { cf = ax[iax] / (dxs[x - 1] + dxs[x]) / dxs[x] * 2.0; dg += cf; od += -v[i - ny] * cf; }
    if (x < nx - 1) { cf = ax[iax + ny] / (dxs[x + 1] + dxs[x]) / dxs[x] * 2.0; dg += cf; od += -v[i + ny] * cf; }
    if (z > 0) { cf = az[i] / (dzs[z - 1] + dzs[z]) / dzs[z] * 2.0; dg += cf; od += -v[i - sl] * cf; }
    if (z < nz - 1) { cf = az[i + sl] / (dzs[z + 1] + dzs[z]) / dzs[z] * 2.0; dg += cf; od += -v[i + sl] * cf; }
    *diag = dg; *off = od;
}

void or_jacobi3d(double* dst, const double* src, const double* f, const double* ax, const double* ay,
                 const double* az, int nx, int ny, int nz, const double* dxs, const double* dys,
                 const double* dzs, double omega) {
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y) {
                long i = y + (long)x * ny + (long)z * nx * ny;
                double dg, od;
                frac_row3d(src, ax, ay, az, nx, ny, nz, dxs, dys, dzs, x, y, z, &dg, &od);
                dst[i] = dg > EPS12 ? (1.0 - omega) * src[i] + omega * (f[i] - od) / dg : 0.0;
            }
}

/* cuWjGetFracRes_3d_n (cuWeightedJacobi3D.cu:1107-1181) */
static void residual3d(double* r, const double* v, const double* f, const double* ax, const double* ay,
                       const double* az, int nx, int ny, int nz, const double* dxs, const double* dys,
                       const double* dzs) {
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y) {
                long i = y + (long)x * ny + (long)z * nx * ny;
                double dg, od;
                frac_row3d(v, ax, ay, az, nx, ny, nz, dxs, dys, dzs, x, y, z, &dg, &od);
                r[i] = dg > EPS12 ? f[i] - (dg * v[i] + od) : 0.0;
            }
}

/* cuWjFrac3D_kernel_n (cuWeightedJacobi3D.cu:1473-1545): 50 volume-scaled Jacobi sweeps */
static void coarsest3d(double* v, const double* f, const double* ax, const double* ay, const double* az,
                       int nx, int ny, int nz, const double* dxs, const double* dys, const double* dzs, double w) {
    long n = (long)nx * ny * nz, sl = (long)nx * ny;
    double* p = (double*)malloc(sizeof(double) * n);
    double* q = (double*)malloc(sizeof(double) * n);
    double* r = (double*)malloc(sizeof(double) * n);
    double* c = (double*)malloc(sizeof(double) * n * 6);
    for (int z = 0; z < nz; ++z)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y) {
                long i = y + (long)x * ny + z * sl;
                long iax = y + (long)x * ny + (long)z * (nx + 1) * ny, iay = y + (long)x * (ny + 1) + (long)z * nx * (ny + 1);
                double vol = dxs[x] * dys[y] * dzs[z], dydz = dys[y] * dzs[z], dxdy = dxs[x] * dys[y], dxdz = dxs[x] * dzs[z];
                int xm = x - 1 < 0 ? 0 : x - 1, xp = x + 1 > nx - 1 ? nx - 1 : x + 1;
                int ym = y - 1 < 0 ? 0 : y - 1, yp = y + 1 > ny - 1 ? ny - 1 : y + 1;
                int zm = z - 1 < 0 ? 0 : z - 1, zp = z + 1 > nz - 1 ? nz - 1 : z + 1;
                c[6 * i + 0] = ax[iax] / (dxs[xm] + dxs[x]) * dydz * 2.0;
                c[6 * i + 1] = ax[iax + ny] / (dxs[xp] + dxs[x]) * dydz * 2.0;
                c[6 * i + 2] = ay[iay] / (dys[ym] + dys[y]) * dxdz * 2.0;
                c[6 * i + 3] = ay[iay + 1] / (dys[yp] + dys[y]) * dxdz * 2.0;
                c[6 * i + 4] = az[i] / (dzs[zm] + dzs[z]) * dxdy * 2.0;
                c[6 * i + 5] = az[i + sl] / (dzs[zp] + dzs[z]) * dxdy * 2.0;
                p[i] = v[i];
                r[i] = f[i] * vol;
            }
    for (int it = 0; it < 50; ++it) {
        for (int z = 0; z < nz; ++z)
            for (int x = 0; x < nx; ++x)
                for (int y = 0; y < ny; ++y) {
                    long i = y + (long)x * ny + z * sl;
                    double od = 0.0, dg = 0.0;
                    if (x > 0) { dg += c[6 * i + 0]; od += -c[6 * i + 0] * p[i - ny]; }
                    if (x < nx - 1) { dg += c[6 * i + 1]; od += -c[6 * i + 1] * p[i + ny]; }
                    if (y > 0) { dg += c[6 * i + 2]; od += -c[6 * i + 2] * p[i - 1]; }
                    if (y < ny - 1) { dg += c[6 * i + 3]; od += -c[6 * i + 3] * p[i + 1]; }
                    if (z > 0) { dg += c[6 * i + 4]; od += -c[6 * i + 4] * p[i - sl]; }
                    if (z < nz - 1) { dg += c[6 * i + 5]; od += -c[6 * i + 5] * p[i + sl]; }
                    q[i] = dg > 0.0 ? (1.0 - w) * p[i] + w * (r[i] - od) / dg : 0.0;
                }
        memcpy(p, q, sizeof(double) * n);
    }
    memcpy(v, p, sizeof(double) * n);
    free(p); free(q); free(r); free(c);
}

static int half_up(int n) { return (n & 1) ? (n >> 1) + 1 : (n >> 1); }

/* face-fraction coarsening along one axis of a 3D array (extents e[3], axis ax):
   main axis: inject even faces (cuRestrict3D.cu:613-668 p1_main, :729-800 p2_main);
   transverse axes: average the (up to) two children (:524-600 p1, :670-727 p2_lesser). */
static double* coarsen_axis(const double* src, const int e[3], int axis, int main_axis, int out_e[3]) {
    int oe[3] = {e[0], e[1], e[2]};
    oe[axis] = main_axis ? (e[axis] >> 1) + 1 : half_up(e[axis]);
    double* dst = (double*)malloc(sizeof(double) * (size_t)oe[0] * oe[1] * oe[2]);
    for (int z = 0; z < oe[2]; ++z)
        for (int x = 0; x < oe[0]; ++x)
            for (int y = 0; y < oe[1]; ++y) {
                int c[3] = {x, y, z};
                int i = c[axis];
                int s0[3] = {x, y, z}, s1[3] = {x, y, z};
                double val;
#define AT(s) src[(s)[1] + (long)(s)[0] * e[1] + (long)(s)[2] * e[0] * e[1]]
                if (main_axis) {
                    int src_i = 2 * i;
                    if ((e[axis] & 1) == 0 && i == oe[axis] - 1) src_i = 2 * i - 1;
                    s0[axis] = src_i;
                    val = AT(s0);
                } else {
                    s0[axis] = 2 * i;
                    if ((e[axis] & 1) == 0) {
                        s1[axis] = 2 * i + 1;
                        val = 0.5 * (AT(s1) + AT(s0));
                    } else {
                        val = 0.5 * AT(s0);
                        if (i < oe[axis] - 1) { s1[axis] = 2 * i + 1; val += 0.5 * AT(s1); }
                        else val *= 2.0;
                    }
                }
#undef AT
                dst[y + (long)x * oe[1] + (long)z * oe[0] * oe[1]] = val;
            }
    out_e[0] = oe[0]; out_e[1] = oe[1]; out_e[2] = oe[2];
    return dst;
}

/* CuRestrict3D::SolveP1Ax/Ay/Az (cuRestrict3D.cu:972-1145): passes x, y, z in order */
static double* coarsen_faces(const double* src, const int cells[3], int face_axis, int out_cells[3]) {
    int e[3] = {cells[0], cells[1], cells[2]};
    e[face_axis] += 1;
    int e1[3], e2[3], e3[3];
    double* t1 = coarsen_axis(src, e, 0, face_axis == 0, e1);
    double* t2 = coarsen_axis(t1, e1, 1, face_axis == 1, e2);
    double* t3 = coarsen_axis(t2, e2, 2, face_axis == 2, e3);
    free(t1); free(t2);
    out_cells[0] = e3[0]; out_cells[1] = e3[1]; out_cells[2] = e3[2];
    out_cells[face_axis] -= 1;
    return t3;
}

/* CuRestrict3D::SolveP1RN(dx,dy,dz) (cuRestrict3D.cu:939-970, kernels :801-882) */
static void restrict_cells3d(double* dst, const double* src, const int fe[3], const double* const d[3]) {
    int e[3] = {fe[0], fe[1], fe[2]};
    double* cur = (double*)malloc(sizeof(double) * (size_t)e[0] * e[1] * e[2]);
    memcpy(cur, src, sizeof(double) * (size_t)e[0] * e[1] * e[2]);
    for (int axis = 0; axis < 3; ++axis) {
        int oe[3] = {e[0], e[1], e[2]};
        oe[axis] = half_up(e[axis]);
        double* nxt = (double*)malloc(sizeof(double) * (size_t)oe[0] * oe[1] * oe[2]);
        for (int z = 0; z < oe[2]; ++z)
            for (int x = 0; x < oe[0]; ++x)
                for (int y = 0; y < oe[1]; ++y) {
                    int s[3] = {x, y, z};
                    int i = s[axis];
                    s[axis] = 2 * i;
                    long i0 = s[1] + (long)s[0] * e[1] + (long)s[2] * e[0] * e[1];
                    double val = d[axis][2 * i] * cur[i0], w = d[axis][2 * i];
                    if (2 * i < e[axis] - 1) {
                        s[axis] = 2 * i + 1;
                        long i1 = s[1] + (long)s[0] * e[1] + (long)s[2] * e[0] * e[1];
                        val += d[axis][2 * i + 1] * cur[i1];
                        w += d[axis][2 * i + 1];
                    }
                    nxt[y + (long)x * oe[1] + (long)z * oe[0] * oe[1]] = val / w;
                }
        free(cur);
        cur = nxt;
        e[0] = oe[0]; e[1] = oe[1]; e[2] = oe[2];
    }
    memcpy(dst, cur, sizeof(double) * (size_t)e[0] * e[1] * e[2]);
    free(cur);
}

typedef struct {
    int n[3];
    double *ax, *ay, *az, *d[3], *v, *f;
} mg3_level;


/* cell-centred trilinear prolongation (weights 3/4, 1/4 per axis; the missing neighbour at a
   wall repeats the parent), added into the fine iterate */
static void prolong_trilinear3d(double* vf, const int nf[3], const double* vc, const int nc[3]) {
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nf[2]; ++z)
        for (int x = 0; x < nf[0]; ++x)
            for (int y = 0; y < nf[1]; ++y) {
                int f3[3] = {x, y, z}, p[3], q[3];
                for (int a = 0; a < 3; ++a) {
                    p[a] = f3[a] / 2;
                    int nb = (f3[a] & 1) ? p[a] + 1 : p[a] - 1;
                    if (nb < 0 || nb >= nc[a]) nb = p[a];
                    q[a] = nb;
                }
                double acc = 0.0;
                for (int cz = 0; cz < 2; ++cz)
                    for (int cx = 0; cx < 2; ++cx)
                        for (int cy = 0; cy < 2; ++cy) {
                            int ix = cx ? q[0] : p[0], iy = cy ? q[1] : p[1], iz = cz ? q[2] : p[2];
                            double w = (cx ? 0.25 : 0.75) * (cy ? 0.25 : 0.75) * (cz ? 0.25 : 0.75);
                            if (nc[2] == 1 && cz) continue;
                            if (nc[2] == 1) w /= 0.75;
                            acc += w * vc[iy + (long)ix * nc[1] + (long)iz * nc[0] * nc[1]];
                        }
                vf[y + (long)x * nf[1] + (long)z * nf[0] * nf[1]] += acc;
            }
}

/* CuMultigridFrac3D::SolveOneVCycle (cuMultigridFrac3D.cu:267-327) */
static void vcycle3d(mg3_level* lv, int nl, int l, int nu1, int nu2, double w, int prolong) {
    mg3_level* c = &lv[l];
    long n = (long)c->n[0] * c->n[1] * c->n[2];
    if (l < nl - 1) {
        double* tmp = (double*)malloc(sizeof(double) * n);
        for (int s = 0; s < nu1; ++s) {
            or_jacobi3d(tmp, c->v, c->f, c->ax, c->ay, c->az, c->n[0], c->n[1], c->n[2], c->d[0], c->d[1], c->d[2], w);
            memcpy(c->v, tmp, sizeof(double) * n);
        }
        residual3d(tmp, c->v, c->f, c->ax, c->ay, c->az, c->n[0], c->n[1], c->n[2], c->d[0], c->d[1], c->d[2]);
        const double* dd[3] = {c->d[0], c->d[1], c->d[2]};
        restrict_cells3d(lv[l + 1].f, tmp, c->n, dd);
        mg3_level* k = &lv[l + 1];
        memset(k->v, 0, sizeof(double) * (size_t)k->n[0] * k->n[1] * k->n[2]);
        vcycle3d(lv, nl, l + 1, nu1, nu2, w, prolong);
        /* CuProlongate3D::SolveAddP1RN (cuProlongate3D.cu:594-617): piecewise-constant add */
        if (prolong == 0) {
            for (int z = 0; z < c->n[2]; ++z)
                for (int x = 0; x < c->n[0]; ++x)
                    for (int y = 0; y < c->n[1]; ++y)
                        c->v[y + (long)x * c->n[1] + (long)z * c->n[0] * c->n[1]] +=
                            k->v[y / 2 + (long)(x / 2) * k->n[1] + (long)(z / 2) * k->n[0] * k->n[1]];
        } else {
            prolong_trilinear3d(c->v, c->n, k->v, k->n);
        }
        for (int s = 0; s < nu2; ++s) {
            or_jacobi3d(tmp, c->v, c->f, c->ax, c->ay, c->az, c->n[0], c->n[1], c->n[2], c->d[0], c->d[1], c->d[2], w);
            memcpy(c->v, tmp, sizeof(double) * n);
        }
        free(tmp);
    } else {
        coarsest3d(c->v, c->f, c->ax, c->ay, c->az, c->n[0], c->n[1], c->n[2], c->d[0], c->d[1], c->d[2], w);
    }
}

static double norm2(const double* a, long n) {
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long i = 0; i < n; ++i) s += a[i] * a[i];
    return s;
}

double or_frac_residual3d(double* r, const double* p, const double* f, const double* ax, const double* ay,
                          const double* az, int nx, int ny, int nz, double dx, double dy, double dz) {
    long n = (long)nx * ny * nz;
    double* rr = r ? r : (double*)malloc(sizeof(double) * n);
    double* dxs = (double*)malloc(sizeof(double) * (nx + ny + nz));
    double *dys = dxs + nx, *dzs = dys + ny;
    for (int i = 0; i < nx; ++i) dxs[i] = dx;
    for (int i = 0; i < ny; ++i) dys[i] = dy;
    for (int i = 0; i < nz; ++i) dzs[i] = dz;
    residual3d(rr, p, f, ax, ay, az, nx, ny, nz, dxs, dys, dzs);
    double res = sqrt(norm2(rr, n)) / sqrt(norm2(f, n));
    free(dxs);
    if (!r) free(rr);
    return res;
}

/* CuMultigridFrac3D ctor (cuMultigridFrac3D.cu:9-134): the coarse hierarchy (ceil halving until the
   smallest extent is 1), face fractions coarsened by SolveP1Ax/Ay/Az, spacings summed pairwise */
static int build_levels3d(mg3_level* lv, const double* ax, const double* ay, const double* az, int nx, int ny,
                          int nz, double dx, double dy, double dz) {
    int nl = 0;
    int n[3] = {nx, ny, nz};
    int mn = nx < ny ? (nx < nz ? nx : nz) : (ny < nz ? ny : nz);
    while (mn > 1 && nl < 32) {
        mg3_level* L = &lv[nl];
        L->n[0] = n[0]; L->n[1] = n[1]; L->n[2] = n[2];
        long cells = (long)n[0] * n[1] * n[2];
        L->v = (double*)calloc(cells, sizeof(double));
        L->f = (double*)calloc(cells, sizeof(double));
        for (int a = 0; a < 3; ++a) L->d[a] = (double*)malloc(sizeof(double) * n[a]);
        if (nl == 0) {
            size_t sx = (size_t)(nx + 1) * ny * nz, sy = (size_t)nx * (ny + 1) * nz, sz = (size_t)nx * ny * (nz + 1);
            L->ax = (double*)malloc(sizeof(double) * sx); memcpy(L->ax, ax, sizeof(double) * sx);
            L->ay = (double*)malloc(sizeof(double) * sy); memcpy(L->ay, ay, sizeof(double) * sy);
            L->az = (double*)malloc(sizeof(double) * sz); memcpy(L->az, az, sizeof(double) * sz);
            for (int i = 0; i < nx; ++i) L->d[0][i] = dx;
            for (int i = 0; i < ny; ++i) L->d[1][i] = dy;
            for (int i = 0; i < nz; ++i) L->d[2][i] = dz;
        } else {
            mg3_level* F = &lv[nl - 1];
            int oc[3];
            L->ax = coarsen_faces(F->ax, F->n, 0, oc);
            L->ay = coarsen_faces(F->ay, F->n, 1, oc);
            L->az = coarsen_faces(F->az, F->n, 2, oc);
            for (int a = 0; a < 3; ++a)
                for (int i = 0; i < n[a]; ++i)
                    L->d[a][i] = F->d[a][2 * i] + (2 * i + 1 < F->n[a] ? F->d[a][2 * i + 1] : 0.0);
        }
        ++nl;
        for (int a = 0; a < 3; ++a) n[a] = half_up(n[a]);
        mn = n[0] < n[1] ? (n[0] < n[2] ? n[0] : n[2]) : (n[1] < n[2] ? n[1] : n[2]);
    }
    return nl;
}

static void free_levels3d(mg3_level* lv, int nl) {
    for (int l = 0; l < nl; ++l) {
        free(lv[l].v); free(lv[l].f); free(lv[l].ax); free(lv[l].ay); free(lv[l].az);
        for (int a = 0; a < 3; ++a) free(lv[l].d[a]);
    }
}

static double rel_residual_l0(mg3_level* lv, double* r) {
    const mg3_level* c = &lv[0];
    long N = (long)c->n[0] * c->n[1] * c->n[2];
    residual3d(r, c->v, c->f, c->ax, c->ay, c->az, c->n[0], c->n[1], c->n[2], c->d[0], c->d[1], c->d[2]);
    return sqrt(norm2(r, N)) / sqrt(norm2(c->f, N));
}

/* CuMultigridFrac3D::Solve (cuMultigridFrac3D.cu:249-265) */
int or_mgfrac3d_solve(double* p, const double* p0, const double* f, const double* ax, const double* ay,
                      const double* az, int nx, int ny, int nz, double dx, double dy, double dz,
                      int ncycles, int nu1, int nu2, double omega, int prolong, double* history) {
    mg3_level lv[32];
    int nl = build_levels3d(lv, ax, ay, az, nx, ny, nz, dx, dy, dz);
    long N = (long)nx * ny * nz;
    if (p0) memcpy(lv[0].v, p0, sizeof(double) * N);
    memcpy(lv[0].f, f, sizeof(double) * N);
    double* r = history ? (double*)malloc(sizeof(double) * N) : NULL;
    for (int c = 0; c < ncycles; ++c) {
        vcycle3d(lv, nl, 0, nu1, nu2, omega, prolong);
        if (history) history[c] = rel_residual_l0(lv, r);
    }
    memcpy(p, lv[0].v, sizeof(double) * N);
    free(r);
    free_levels3d(lv, nl);
    return nl;
}

/* ------------------------------------------- index-sparse fractional multigrid 3D ---- */
/* CuBoundSelector::SelectByFrac (cuBoundSelector.cu:4-32): a cell takes part in the index-sparse
   cycle when any of its six face fractions is >= 1e-12 (boundary faces included); InitIndex
   (cuMultigridFrac3D.cu:189-229) lists those cells per level. */
static unsigned char* active_cells3d(const mg3_level* c, long* count) {
    const int nx = c->n[0], ny = c->n[1], nz = c->n[2];
    const long sl = (long)nx * ny;
    unsigned char* a = (unsigned char*)malloc((size_t)sl * nz);
    long cnt = 0;
    for (int z = 0; z < nz; ++z)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y) {
                long i = y + (long)x * ny + z * sl;
                long iax = y + (long)x * ny + (long)z * (nx + 1) * ny, iay = y + (long)x * (ny + 1) + (long)z * nx * (ny + 1);
                int on = !(c->ax[iax] < EPS12 && c->ax[iax + ny] < EPS12 && c->ay[iay] < EPS12 && c->ay[iay + 1] < EPS12 &&
                           c->az[i] < EPS12 && c->az[i + sl] < EPS12);
                a[i] = (unsigned char)on;
                cnt += on;
            }
    *count = cnt;
    return a;
}

/* CuWeightedJacobi3D::SolveFrac with an index list (cuWeightedJacobi3D.cu:2821-2897, 2979-3011):
   the sweep updates the listed cells only; every other cell keeps its value */
static void jacobi3d_index(mg3_level* c, const unsigned char* act, int sweeps, double w, double* tmp) {
    const long n = (long)c->n[0] * c->n[1] * c->n[2];
    for (int s = 0; s < sweeps; ++s) {
        memcpy(tmp, c->v, sizeof(double) * n);
#pragma omp parallel for schedule(static)
        for (int z = 0; z < c->n[2]; ++z)
            for (int x = 0; x < c->n[0]; ++x)
                for (int y = 0; y < c->n[1]; ++y) {
                    long i = y + (long)x * c->n[1] + (long)z * c->n[0] * c->n[1];
                    if (!act[i]) continue;
                    double dg, od;
                    frac_row3d(c->v, c->ax, c->ay, c->az, c->n[0], c->n[1], c->n[2], c->d[0], c->d[1], c->d[2], x, y, z,
                               &dg, &od);
                    tmp[i] = dg > EPS12 ? (1.0 - w) * c->v[i] + w * (c->f[i] - od) / dg : 0.0;
                }
        memcpy(c->v, tmp, sizeof(double) * n);
    }
}

/* SolveOneVCycle_index (cuMultigridFrac3D.cu:366-420).  R is the residual workspace shared by all
   levels (the reference's "mg3d" buffer): the residual kernel (cuWjGetFracRes_3d_n with an index,
   cuWeightedJacobi3D.cu:3013-3090) writes the listed cells of the level only, and the restriction
   (cuRestrict3D_p1_dx_whole, cuRestrict3D.cu:1146-1193) reads all children of each listed coarse
   cell, so an unlisted child contributes whatever R last held at its position (zero until some
   level wrote there).  Post-smoothing runs nu1 sweeps, as the reference passes nu1 there. */
static void vcycle3d_index(mg3_level* lv, unsigned char* const* act, const long* cnt, int nl, int l, int nu1,
                           double w, double* R, double* tmp) {
    mg3_level* c = &lv[l];
    const int nx = c->n[0], ny = c->n[1], nz = c->n[2];
    if (l < nl - 1 && cnt[l + 1] > 0) {
        jacobi3d_index(c, act[l], nu1, w, tmp);
#pragma omp parallel for schedule(static)
        for (int z = 0; z < nz; ++z)
            for (int x = 0; x < nx; ++x)
                for (int y = 0; y < ny; ++y) {
                    long i = y + (long)x * ny + (long)z * nx * ny;
                    if (!act[l][i]) continue;
                    double dg, od;
                    frac_row3d(c->v, c->ax, c->ay, c->az, nx, ny, nz, c->d[0], c->d[1], c->d[2], x, y, z, &dg, &od);
                    R[i] = dg > EPS12 ? c->f[i] - (dg * c->v[i] + od) : 0.0;
                }
        mg3_level* k = &lv[l + 1];
        const int cx = k->n[0], cy = k->n[1], cz = k->n[2];
#pragma omp parallel for schedule(static)
        for (int z = 0; z < cz; ++z)
            for (int x = 0; x < cx; ++x)
                for (int y = 0; y < cy; ++y) {
                    long ci = y + (long)x * cy + (long)z * cx * cy;
                    if (!act[l + 1][ci]) continue;
                    int xs = 2 * x, ys = 2 * y, zs = 2 * z;
                    int hx = xs < nx - 1, hy = ys < ny - 1, hz = zs < nz - 1;
                    double wxl = c->d[0][xs], wyl = c->d[1][ys], wzl = c->d[2][zs];
                    double wxr = hx ? c->d[0][xs + 1] : 0.0, wyr = hy ? c->d[1][ys + 1] : 0.0, wzr = hz ? c->d[2][zs + 1] : 0.0;
                    long ox = hx ? ny : 0, oy = hy ? 1 : 0, oz = hz ? (long)nx * ny : 0;
                    long s0 = ys + (long)xs * ny + (long)zs * nx * ny;
                    double val = wxl * wyl * wzl * R[s0];
                    val += wxl * wyr * wzl * R[s0 + oy];
                    val += wxr * wyl * wzl * R[s0 + ox];
                    val += wxr * wyr * wzl * R[s0 + oy + ox];
                    s0 += oz;
                    val += wxl * wyl * wzr * R[s0];
                    val += wxl * wyr * wzr * R[s0 + oy];
                    val += wxr * wyl * wzr * R[s0 + ox];
                    val += wxr * wyr * wzr * R[s0 + oy + ox];
                    k->f[ci] = val / ((wxl + wxr) * (wyl + wyr) * (wzl + wzr));
                }
        memset(k->v, 0, sizeof(double) * (size_t)cx * cy * cz);
        vcycle3d_index(lv, act, cnt, nl, l + 1, nu1, w, R, tmp);
        /* cuProlongate3D_p1_whole_add (cuProlongate3D.cu:619-640): listed cells only */
        for (int z = 0; z < nz; ++z)
            for (int x = 0; x < nx; ++x)
                for (int y = 0; y < ny; ++y) {
                    long i = y + (long)x * ny + (long)z * nx * ny;
                    if (act[l][i]) c->v[i] += k->v[y / 2 + (long)(x / 2) * cy + (long)(z / 2) * cx * cy];
                }
        jacobi3d_index(c, act[l], nu1, w, tmp);
    } else {
        coarsest3d(c->v, c->f, c->ax, c->ay, c->az, nx, ny, nz, c->d[0], c->d[1], c->d[2], w);
    }
}

/* CuMultigridFrac3D::Solve_index (cuMultigridFrac3D.cu:347-364) from a fresh residual workspace;
   counts (may be NULL) receives the listed cells per level.  nu2 is accepted and not used. */
int or_mgfrac3d_solve_index(double* p, const double* p0, const double* f, const double* ax, const double* ay,
                            const double* az, int nx, int ny, int nz, double dx, double dy, double dz, int ncycles,
                            int nu1, int nu2, double omega, double* history, long* counts) {
    (void)nu2;
    mg3_level lv[32];
    int nl = build_levels3d(lv, ax, ay, az, nx, ny, nz, dx, dy, dz);
    unsigned char* act[32];
    long cnt[32];
    for (int l = 0; l < nl; ++l) {
        act[l] = active_cells3d(&lv[l], &cnt[l]);
        if (counts) counts[l] = cnt[l];
    }
    long N = (long)nx * ny * nz;
    if (p0) memcpy(lv[0].v, p0, sizeof(double) * N);
    memcpy(lv[0].f, f, sizeof(double) * N);
    double* R = (double*)calloc(N, sizeof(double));
    double* tmp = (double*)malloc(sizeof(double) * N);
    for (int c = 0; c < ncycles; ++c) {
        vcycle3d_index(lv, act, cnt, nl, 0, nu1, omega, R, tmp);
        if (history) history[c] = rel_residual_l0(lv, tmp);
    }
    memcpy(p, lv[0].v, sizeof(double) * N);
    free(R); free(tmp);
    for (int l = 0; l < nl; ++l) free(act[l]);
    free_levels3d(lv, nl);
    return nl;
}

/* ------------------------------------------------------- fractional multigrid 2D ---- */
/* cuWeightedJacobi_frac_n (cuWeightedJacobi.cu:292-347) */
static inline void frac_row2d(const double* v, const double* ax, const double* ay, int nx, int ny,
                              const double* dxs, const double* dys, int x, int y, double* diag, double* off) {
    long i = y + (long)x * ny, iay = y + (long)x * (ny + 1);
    double dg = 0.0, od = 0.0, cf;
    if (y > 0) { cf = ay[iay] / (dys[y - 1] + dys[y]) / dys[y] * 2.0; dg += cf; od += -cf * v[i - 1]; }
    if (y < ny - 1) { cf = ay[iay + 1] / (dys[y + 1] + dys[y]) / dys[y] * 2.0; dg += cf; od += -cf * v[i + 1]; }
    if (x > 0) { cf = ax[i] / (dxs[x - 1] + dxs[x]) / dxs[x] * 2.0; dg += cf; od += -v[i - ny] * cf; }
    if (x < nx - 1) { cf = ax[i + ny] / (dxs[x + 1] + dxs[x]) / dxs[x] * 2.0; dg += cf; od += -v[i + ny] * cf; }
    *diag = dg; *off = od;
}

static void jacobi2d(double* dst, const double* src, const double* f, const double* ax, const double* ay, int nx,
                     int ny, const double* dxs, const double* dys, double w) {
#pragma omp parallel for schedule(static)
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y) {
            long i = y + (long)x * ny;
            double dg, od;
            frac_row2d(src, ax, ay, nx, ny, dxs, dys, x, y, &dg, &od);
            dst[i] = dg > EPS12 ? (1.0 - w) * src[i] + w * (f[i] - od) / dg : 0.0;
        }
}

static void residual2d(double* r, const double* v, const double* f, const double* ax, const double* ay, int nx,
                       int ny, const double* dxs, const double* dys) {
#pragma omp parallel for schedule(static)
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y) {
            long i = y + (long)x * ny;
            double dg, od;
            frac_row2d(v, ax, ay, nx, ny, dxs, dys, x, y, &dg, &od);
            r[i] = dg > EPS12 ? f[i] - (dg * v[i] + od) : 0.0;
        }
}

typedef struct {
    int n[2];
    double *ax, *ay, *d[2], *v, *f;
} mg2_level;

static void vcycle2d(mg2_level* lv, int nl, int l, int nu1, int nu2, double w, int prolong) {
    mg2_level* c = &lv[l];
    long n = (long)c->n[0] * c->n[1];
    double* tmp = (double*)malloc(sizeof(double) * n);
    if (l < nl - 1) {
        for (int s = 0; s < nu1; ++s) {
            jacobi2d(tmp, c->v, c->f, c->ax, c->ay, c->n[0], c->n[1], c->d[0], c->d[1], w);
            memcpy(c->v, tmp, sizeof(double) * n);
        }
        residual2d(tmp, c->v, c->f, c->ax, c->ay, c->n[0], c->n[1], c->d[0], c->d[1]);
        mg2_level* k = &lv[l + 1];
        /* CuRestriction2D::SolveP1RN(dx,dy): x pass then y pass, spacing-weighted */
        int e[3] = {c->n[0], c->n[1], 1};
        double one = 1.0;
        const double* dd[3] = {c->d[0], c->d[1], &one};
        restrict_cells3d(k->f, tmp, e, dd);
        memset(k->v, 0, sizeof(double) * (size_t)k->n[0] * k->n[1]);
        vcycle2d(lv, nl, l + 1, nu1, nu2, w, prolong);
        if (prolong == 0) {
            for (int x = 0; x < c->n[0]; ++x)
                for (int y = 0; y < c->n[1]; ++y) c->v[y + (long)x * c->n[1]] += k->v[y / 2 + (long)(x / 2) * k->n[1]];
        } else {
            int nf3[3] = {c->n[0], c->n[1], 1}, nc3[3] = {k->n[0], k->n[1], 1};
            prolong_trilinear3d(c->v, nf3, k->v, nc3);
        }
        for (int s = 0; s < nu2; ++s) {
            jacobi2d(tmp, c->v, c->f, c->ax, c->ay, c->n[0], c->n[1], c->d[0], c->d[1], w);
            memcpy(c->v, tmp, sizeof(double) * n);
        }
    } else {
        /* coarsest: 10 ordinary weighted-Jacobi sweeps (cuMultigridFrac2D.cu:205-207) */
        for (int s = 0; s < 10; ++s) {
            jacobi2d(tmp, c->v, c->f, c->ax, c->ay, c->n[0], c->n[1], c->d[0], c->d[1], w);
            memcpy(c->v, tmp, sizeof(double) * n);
        }
    }
    free(tmp);
}

double or_frac_residual2d(double* r, const double* p, const double* f, const double* ax, const double* ay,
                          int nx, int ny, double dx, double dy) {
    long n = (long)nx * ny;
    double* rr = r ? r : (double*)malloc(sizeof(double) * n);
    double* dxs = (double*)malloc(sizeof(double) * (nx + ny));
    double* dys = dxs + nx;
    for (int i = 0; i < nx; ++i) dxs[i] = dx;
    for (int i = 0; i < ny; ++i) dys[i] = dy;
    residual2d(rr, p, f, ax, ay, nx, ny, dxs, dys);
    double res = sqrt(norm2(rr, n)) / sqrt(norm2(f, n));
    free(dxs);
    if (!r) free(rr);
    return res;
}

int or_mgfrac2d_solve(double* p, const double* p0, const double* f, const double* ax, const double* ay,
                      int nx, int ny, double dx, double dy, int ncycles, int nu1, int nu2, double omega,
                      int prolong, double* history) {
    mg2_level lv[32];
    int nl = 0;
    int n[2] = {nx, ny};
    int mn = nx < ny ? nx : ny;
    while (mn > 1 && nl < 32) {
        mg2_level* L = &lv[nl];
        L->n[0] = n[0]; L->n[1] = n[1];
        long cells = (long)n[0] * n[1];
        L->v = (double*)calloc(cells, sizeof(double));
        L->f = (double*)calloc(cells, sizeof(double));
        for (int a = 0; a < 2; ++a) L->d[a] = (double*)malloc(sizeof(double) * n[a]);
        if (nl == 0) {
            size_t sx = (size_t)(nx + 1) * ny, sy = (size_t)nx * (ny + 1);
            L->ax = (double*)malloc(sizeof(double) * sx); memcpy(L->ax, ax, sizeof(double) * sx);
            L->ay = (double*)malloc(sizeof(double) * sy); memcpy(L->ay, ay, sizeof(double) * sy);
            for (int i = 0; i < nx; ++i) L->d[0][i] = dx;
            for (int i = 0; i < ny; ++i) L->d[1][i] = dy;
        } else {
            mg2_level* F = &lv[nl - 1];
            int c3[3] = {F->n[0], F->n[1], 1}, oc[3];
            L->ax = coarsen_faces(F->ax, c3, 0, oc);
            L->ay = coarsen_faces(F->ay, c3, 1, oc);
            for (int a = 0; a < 2; ++a)
                for (int i = 0; i < n[a]; ++i)
                    L->d[a][i] = F->d[a][2 * i] + (2 * i + 1 < F->n[a] ? F->d[a][2 * i + 1] : 0.0);
        }
        ++nl;
        n[0] = half_up(n[0]); n[1] = half_up(n[1]);
        mn = n[0] < n[1] ? n[0] : n[1];
    }
    long N = (long)nx * ny;
    if (p0) memcpy(lv[0].v, p0, sizeof(double) * N);
    memcpy(lv[0].f, f, sizeof(double) * N);
    double* r = history ? (double*)malloc(sizeof(double) * N) : NULL;
    for (int c = 0; c < ncycles; ++c) {
        vcycle2d(lv, nl, 0, nu1, nu2, omega, prolong);
        if (history) {
            residual2d(r, lv[0].v, lv[0].f, lv[0].ax, lv[0].ay, nx, ny, lv[0].d[0], lv[0].d[1]);
            history[c] = sqrt(norm2(r, N)) / sqrt(norm2(lv[0].f, N));
        }
    }
    memcpy(p, lv[0].v, sizeof(double) * N);
    free(r);
    for (int l = 0; l < nl; ++l) {
        free(lv[l].v); free(lv[l].f); free(lv[l].ax); free(lv[l].ay);
        free(lv[l].d[0]); free(lv[l].d[1]);
    }
    return nl;
}

/* --------------------------------------------------------------------- DST-I ---- */
/* orthonormal DST-I along one axis, in place: (S v)_k = sqrt(2/(n+1)) sum_j v_j sin(pi (j+1)(k+1)/(n+1)) */
static void dst1_axis(double* a, const int e[3], int axis) {
    int n = e[axis];
    double s = sqrt(2.0 / (n + 1));
    double* tab = (double*)malloc(sizeof(double) * (size_t)n * n);
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j) tab[k * n + j] = s * sin(M_PI * (double)(j + 1) * (double)(k + 1) / (n + 1));
    long stride = axis == 1 ? 1 : (axis == 0 ? e[1] : (long)e[0] * e[1]);
    int o1 = axis == 0 ? 1 : 0, o2 = axis == 2 ? 1 : 2;
#pragma omp parallel for collapse(2) schedule(static)
    for (int u = 0; u < e[o1]; ++u)
        for (int w = 0; w < e[o2]; ++w) {
            int c[3] = {0, 0, 0};
            c[o1] = u; c[o2] = w;
            long base = c[1] + (long)c[0] * e[1] + (long)c[2] * e[0] * e[1];
            double* in = (double*)malloc(sizeof(double) * n);
            for (int j = 0; j < n; ++j) in[j] = a[base + j * stride];
            for (int k = 0; k < n; ++k) {
                double acc = 0.0;
                for (int j = 0; j < n; ++j) acc += tab[k * n + j] * in[j];
                a[base + k * stride] = acc;
            }
            free(in);
        }
    free(tab);
}

void or_dst3d_poisson(double* p, const double* f, int nx, int ny, int nz, double dx, double dy, double dz) {
    (void)dz;
    int e[3] = {nx, ny, nz};
    long N = (long)nx * ny * nz;
    memcpy(p, f, sizeof(double) * N);
    dst1_axis(p, e, 0);
    dst1_axis(p, e, 1);
    dst1_axis(p, e, 2);
    for (int z = 0; z < nz; ++z)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y) {
                double mu = 2.0 - 2.0 * cos((x + 1) * M_PI / (nx + 1));
                double nu = 2.0 - 2.0 * cos((y + 1) * M_PI / (ny + 1));
                double ku = 2.0 - 2.0 * cos((z + 1) * M_PI / (nz + 1));
                p[y + (long)x * ny + (long)z * nx * ny] *= dx * dy / (mu + nu + ku);
            }
    dst1_axis(p, e, 2);
    dst1_axis(p, e, 1);
    dst1_axis(p, e, 0);
}
