// wp_dwt.cu -- full-depth multilevel CDF3.7 / CDF4.6 lifting transforms along one axis.
//
// Reference behaviour: CuWHHDForward::Solve1D and the cuWHHDForward_{y,x,z}_ml /
// cuWHHDBackward_{y,x,z}_ml kernels (cuWHHDForward.cu:5-742, 1122-1253) with the step functions
// and boundary rules of cuWaveletCompute.cuh (CDF3.7: :876-900, :944-964, reflection :180-228,
// :600-631; CDF4.6: :925-942, :983-1002, reflection :336-375, :716-752; base matrices :773-874).
// Output layout (Mallat order): [base (4+ext) | d level 2 (4) | d level 3 (8) | ... | d level L-1 (n/2)].
//
// B200 design: one CTA owns a tile of C whole lines (C = 32/16/8/4 columns) staged in shared
// memory as S[position][column] (column pitch C+1 so both the y-contiguous load and the
// column-parallel lifting are bank-conflict free).  All levels run on chip; global memory is
// read once and written once per pass, coalesced along y for every axis (for the x and z axes
// the C columns are C consecutive y; for the y axis the tile is C consecutive whole lines,
// one contiguous span).  Each thread lifts a chunk of 8 coefficient pairs per level from a
// register window of 8+8 pairs (4-pair halo each side), so the lifting taps never touch
// shared memory twice and need no shuffles.
#include "wp_common.cuh"

#include <cstdio>
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace {

// Coefficient pairs per thread per level: 8, or 9 for CDF4.6, whose lines have 2^L + 1 samples in the
// recovery: the 2^(L-1) + 1 approximations of the top level then split into 15 chunks (two rounds of
// a 256-thread tile of 32 columns) instead of 17 (three rounds, the last one eighth full).
__host__ __device__ constexpr int ch_of(int wav) {
    return (wav == WP_ID_CDF4_6 || wav == WP_ID_CDF4_4 || wav == WP_ID_CDF2_6 || wav == WP_ID_CDF2_8 ||
            wav == WP_ID_CDF2_0) ? 9 : 8;
}
constexpr int NT = 256;      // threads per CTA

// lifting constants (cuWaveletCompute.cuh:13-23, :139-148)
#define WP_SQ2 1.41421356237309504880168872420969807856967187537694
#define WP_SQ2_D 1.414213562373095048801
struct K37 {
    static constexpr double fu1 = -1.0 / 3.0;
    static constexpr double fp0 = -3.0 / 8.0, fp1 = -9.0 / 8.0;
    static constexpr double q0 = -0.003797743055556, q1 = 0.032552083333333, q2 = -0.137044270833333,
                            q3 = 0.444444444444444, q4 = 0.137044270833333, q5 = -0.032552083333333,
                            q6 = 0.003797743055556;
    static constexpr double scl0 = 3.0 / 1.414213562373095048801, scl1 = 1.414213562373095048801 / 3.0;
};
// CDF3.5 (cuWaveletCompute.cuh:15 RSW_Q5_fu_2): CDF3.7's first update, predict and scaling with a
// 5-tap second update, written in CDF3.7's 7-tap form with zero outer taps
struct K35 : K37 {
    // q_i weighs the detail at offset 3 - i (RSW_Q5_fu_2[j] weighs offset 2 - j)
    static constexpr double q0 = 0.0, q1 = 5.0 / 288, q2 = -34.0 / 288, q3 = 128.0 / 288, q4 = 34.0 / 288,
                            q5 = -5.0 / 288, q6 = 0.0;
};
template <int WAV>
struct K3 : K37 {};
template <>
struct K3<WP_ID_CDF3_5> : K35 {};
__host__ __device__ constexpr bool is_q3(int w) { return w == WP_ID_CDF3_7 || w == WP_ID_CDF3_5; }
__host__ __device__ constexpr bool is_c4(int w) { return w == WP_ID_CDF4_6 || w == WP_ID_CDF4_4; }
__host__ __device__ constexpr bool is_l2(int w) { return w == WP_ID_CDF2_6 || w == WP_ID_CDF2_8; }
// CDF2.6 / CDF2.8 (cuWaveletCompute.cuh:72-81): a predict from the two neighbouring approximations and
// one update from NT details at offsets -NT/2 .. NT/2 - 1; u[i] weighs offset NT/2 - 1 - i
template <int WAV>
struct K2 {
    static constexpr double fp0 = -0.5, fp1 = -0.5;
    static constexpr double scl0 = WP_SQ2_D, scl1 = 1.0 / WP_SQ2_D;
    static constexpr int NTAP = WAV == WP_ID_CDF2_6 ? 6 : 8;
    __host__ __device__ static constexpr double u(int i) {
        return WAV == WP_ID_CDF2_6
                   ? (i == 0 ? 0.009765625 : i == 1 ? -0.076171875 : i == 2 ? 0.31640625 : i == 3 ? 0.31640625
                      : i == 4 ? -0.076171875 : 0.009765625)
                   : (i == 0 ? -0.002136230468750 : i == 1 ? 0.020446777343750 : i == 2 ? -0.095397949218750
                      : i == 3 ? 0.327087402343750 : i == 4 ? 0.327087402343750 : i == 5 ? -0.095397949218750
                      : i == 6 ? 0.020446777343750 : -0.002136230468750);
    }
};
// The short families (cuWaveletCompute.cuh:6-11, 1397-1556): CDF2.0 is CDF2.x's predict alone with the
// detail's scale negated; CDF1.1 the Haar step (d - a, then a + d / 2); CDF1.7 the Haar predict and a
// 7-tap update, t7(i) weighing the detail at offset 3 - i
__host__ __device__ constexpr bool is_t1(int w) { return w == WP_ID_CDF1_1 || w == WP_ID_CDF1_7; }
// boundary rules: CDF1.x take CDF3.5's (cuWT_CDF3_5_*), CDF2.0 CDF2.6's (cuWT_CDF2_6_*)
__host__ __device__ constexpr bool q3_rules(int w) { return is_q3(w) || is_t1(w); }
__host__ __device__ constexpr bool l2_rules(int w) { return is_l2(w) || w == WP_ID_CDF2_0; }
struct KT {
    static constexpr double fp = -1.0, fu = 0.5;
    static constexpr double scl0 = WP_SQ2_D, scl1 = 1.0 / 1.41421356237309504, scl7_1 = -1.0 / 1.41421356237309504;
    __host__ __device__ static constexpr double t7(int i) {
        return i == 0 ? -0.002441406250000 : i == 1 ? 0.021484375000000 : i == 2 ? -0.098144531250000
             : i == 3 ? 0.5 : i == 4 ? 0.098144531250000 : i == 5 ? -0.021484375000000 : 0.002441406250000;
    }
};
// CDF4.4's second update (RSW_C4_fu_2): d4_i weighs offset 1 - i
struct K44 {
    static constexpr double d0 = -0.03906250, d1 = 0.22656250, d2 = 0.22656250, d3 = -0.03906250;
};
struct K46 {
    static constexpr double fu1_0 = -0.25, fu1_1 = -0.25;
    static constexpr double fp0 = -1.0, fp1 = -1.0;
    static constexpr double c0 = 0.008544921875000, c1 = -0.064697265625000, c2 = 0.243652343750000,
                            c3 = 0.243652343750000, c4 = -0.064697265625000, c5 = 0.008544921875000;
    static constexpr double scl0 = 2.0 * WP_SQ2, scl1 = -1.0 / (2.0 * WP_SQ2);
    static constexpr double scli0 = 1.0 / (2.0 * WP_SQ2), scli1 = -(2.0 * WP_SQ2);
};

// base-level matrices, row-major, in this order: 37n, 37d, 46n, 46d (forward), then inverses
__constant__ double c_base37[4][16];
__constant__ double c_base35[4][16];
__constant__ double c_base46[4][25];
// CDF4.4: forward n, forward d, inverse n, inverse d; CDF2.6 / CDF2.8: forward n, d, z, inverse n, d, z
__constant__ double c_base44[4][25];
__constant__ double c_base26[6][25];
__constant__ double c_base28[6][25];
// CDF2.0: forward, inverse (one matrix for 'n' and 'd'); CDF1.1: forward, inverse; CDF1.7: forward n, d,
// inverse n, d
__constant__ double c_base20[2][25];
__constant__ double c_base11[2][16];
__constant__ double c_base17[4][16];
// RSW_20_L10 / RSW_i20_L10, RSW_11_L10 / RSW_i11_L10, RSW_T{N,D}7_L10 / RSW_iT{N,D}7_L10
// (cuWaveletCompute.cuh:1398-1411, 1438-1449, 1479-1502)
const double h_base20[2][25] = {
    {2.0, 0, 0, 0, 0, 0, 0, 0, 0, 2.0, 0.5, 0, -1.0, 0, 0.5, 0.353553390593274, -0.707106781186547, 0.353553390593274, 0, 0, 0, 0, 0.353553390593274, -0.707106781186547, 0.353553390593274},
    {0.5, 0, 0, 0, 0, 0.375, 0.125, -0.5, -1.414213562373095, 0, 0.25, 0.25, -1.0, 0, 0, 0.125, 0.375, -0.5, 0, -1.414213562373095, 0, 0.5, 0, 0, 0}};
const double h_base11[2][16] = {
    {0.5, 0.5, 0.5, 0.5, -0.5, -0.5, 0.5, 0.5, -0.707106781186548, 0.707106781186548, 0, 0, 0, 0, -0.707106781186548, 0.707106781186548},
    {0.5, -0.5, -0.707106781186547, 0, 0.5, -0.5, 0.707106781186547, 0, 0.5, 0.5, 0, -0.707106781186547, 0.5, 0.5, 0, 0.707106781186547}};
const double h_base17[4][16] = {
    {0.5, 0.5, 0.5, 0.5, 0.69140625, 0.30859375, -0.30859375, -0.69140625, 0.707106781186548, -0.707106781186548, 0, 0, 0, 0, 0.707106781186548, -0.707106781186548},
    {0.30859375, 0.69140625, 0.69140625, 0.30859375, 0.5, 0.5, -0.5, -0.5, 0.707106781186548, -0.707106781186548, 0, 0, 0, 0, 0.707106781186548, -0.707106781186548},
    {0.5, 0.5, 0.571762123850060, -0.135344657336488, 0.5, 0.5, -0.842451438523035, -0.135344657336488, 0.5, -0.5, 0.135344657336488, 0.842451438523035, 0.5, -0.5, 0.135344657336488, -0.571762123850060},
    {0.5, 0.5, 0.842451438523035, -0.135344657336488, 0.5, 0.5, -0.571762123850060, -0.135344657336488, 0.5, -0.5, 0.135344657336488, 0.571762123850060, 0.5, -0.5, 0.135344657336488, -0.842451438523035}};

const double h_base37[4][16] = {
    {0.500000000000000, 0.500000000000000, 0.500000000000000, 0.500000000000000, -0.399902343750000,
     -0.200195312500000, 0.200195312500000, 0.399902343750000, -0.353553390593274, 0.530330085889911,
     -0.176776695296637, 0, 0, 0.176776695296637, -0.530330085889911, 0.353553390593274},
    {0.800781250000000, 1.599609375000000, 1.599609375000000, 0.800781250000000, -1.000000000000000,
     -1.000000000000000, 1.000000000000000, 1.000000000000000, -0.707106781186548, 0.530330085889911,
     -0.176776695296637, 0, 0, 0.176776695296637, -0.530330085889911, 0.707106781186548},
    {0.500000000000000, -1.000000000000000, -0.990225707247567, 0.423987855125528, 0.500000000000000,
     -0.500000000000000, 1.272654099342585, -0.141559463030510, 0.500000000000000, 0.500000000000000,
     0.141559463030510, -1.272654099342585, 0.500000000000000, 1.000000000000000, -0.423987855125528,
     0.990225707247567},
    {0.125000000000000, -0.250000000000000, -0.919100708749311, 0.211993927562764, 0.250000000000000,
     -0.250000000000000, 0.636672316654294, 0.070434464532254, 0.250000000000000, 0.250000000000000,
     -0.070434464532254, -0.636672316654294, 0.125000000000000, 0.250000000000000, -0.211993927562764,
     0.919100708749311}};
// CDF3.5 base-level matrices (cuWaveletCompute.cuh:34-45, 60-71): forward n, forward d, inverse n, inverse d
const double h_base35[4][16] = {
    {0.5, 0.5, 0.5, 0.5, -0.3828125, -0.234375, 0.234375, 0.3828125, -0.353553390593274, 0.530330085889911,
     -0.176776695296637, 0, 0, 0.176776695296637, -0.530330085889911, 0.353553390593274},
    {0.937499999999999, 1.53125, 1.53125, 0.9375, -1.0, -1.0, 1.0, 1.0, -0.707106781186548, 0.530330085889911,
     -0.176776695296637, 0, 0, 0.176776695296637, -0.530330085889911, 0.707106781186548},
    {0.5, -1.0, -1.038563084867742, 0.375650477505353, 0.5, -0.5, 1.248485410532498, -0.165728151840597, 0.5, 0.5,
     0.165728151840597, -1.248485410532498, 0.5, 1.0, -0.375650477505353, 1.038563084867742},
    {0.125, -0.25, -0.894932019939224, 0.187825238752677, 0.25, -0.25, 0.685009694274468, 0.02209708691208, 0.25,
     0.25, -0.02209708691208, -0.685009694274468, 0.125, 0.25, -0.187825238752677, 0.894932019939224}};
// base-level matrices of CDF4.4 and CDF2.6 / CDF2.8 (cuWaveletCompute.cuh:94-137, 150-177, 799-845:
// RSW_CN4_L10, RSW_CD4_L10, RSW_L{N,D,Z}{6,8}_L10 and their inverses)
const double h_base44[4][25] = {
    {2.125, 1.6875, 0.5, -0.6875, -1.625, -1.625, -0.6875, 0.5, 1.6875, 2.125, 1.0, 0, -2.0, 0, 1.0, 0.353553390593274, -0.618718433538229, 0.353553390593274, -0.088388347648318, 0, 0, -0.088388347648318, 0.353553390593274, -0.618718433538229, 0.353553390593274},
    {2.05078125, 0, 0, 0, 0, 0, 0, 0, 0, 2.05078125, 0.734375, -0.1484375, -0.46875, -0.1484375, 0.734375, 0.353553390593274, -0.441941738241592, 0.353553390593274, -0.088388347648318, 0, 0, -0.088388347648318, 0.353553390593274, -0.441941738241592, 0.353553390593274},
    {0.34375, 0.15625, 0.25, 0.773398041922786, -0.066291260736239, 0.3125, 0.1875, 0, -1.016465997955662, 0.309359216769115, 0.25, 0.25, -0.25, 0.353553390593274, 0.353553390593274, 0.1875, 0.3125, 0, 0.309359216769115, -1.016465997955662, 0.15625, 0.34375, 0.25, -0.066291260736239, 0.773398041922786},
    {0.125, 0, 0, 0, 0, 0.25, 0.125, -1.0, -2.077126169735483, 0.751300955010707, 0.21875, 0.21875, -1.5, 0.419844651329513, 0.419844651329513, 0.125, 0.25, -1.0, 0.751300955010707, -2.077126169735483, 0, 0.125, 0, 0, 0}};
const double h_base26[6][25] = {
    {0.8671875, 1.265625, 0.5, -0.265625, -0.3671875, -0.3671875, -0.265625, 0.5, 1.265625, 0.8671875, -0.5, 0, 1.0, 0, -0.5, -0.353553390593274, 0.707106781186547, -0.353553390593274, 0, 0, 0, 0, -0.353553390593274, 0.707106781186547, -0.353553390593274},
    {2.0, 0, 0, 0, 0, 0, 0, 0, 0, 2.0, -0.69140625, 0.3828125, 0.6171875, 0.3828125, -0.69140625, -0.353553390593274, 0.707106781186547, -0.353553390593274, 0, 0, 0, 0, -0.353553390593274, 0.707106781186547, -0.353553390593274},
    {0.8671875, 0.6328125, 0.25, -0.1328125, -0.3671875, -0.3671875, -0.1328125, 0.25, 0.6328125, 0.8671875, -1.0, 0, 1.0, 0, -1.0, -0.707106781186547, 0.707106781186547, -0.353553390593274, 0, 0, 0, 0, -0.353553390593274, 0.707106781186547, -0.707106781186547},
    {0.5, 0, -0.5, -0.894932019939224, 0.187825238752677, 0.375, 0.125, 0, 0.789970857106846, -0.082864075920299, 0.25, 0.25, 0.5, -0.353553390593274, -0.353553390593274, 0.125, 0.375, 0, -0.082864075920299, 0.789970857106846, 0, 0.5, -0.5, 0.187825238752677, -0.894932019939224},
    {0.5, 0, 0, 0, 0, 0.375, 0.125, 0.5, 1.143524247700120, -0.270689314672975, 0.25, 0.25, 1.0, -0.541378629345950, -0.541378629345950, 0.125, 0.375, 0.5, -0.270689314672975, 1.143524247700120, 0, 0.5, 0, 0, 0},
    {0.5, 0, -0.25, -0.447466009969612, 0.093912619376338, 0.75, 0.25, 0, 0.789970857106846, -0.082864075920299, 0.5, 0.5, 0.5, -0.353553390593274, -0.353553390593274, 0.25, 0.75, 0, -0.082864075920299, 0.789970857106846, 0, 0.5, -0.25, 0.093912619376338, -0.447466009969612}};
const double h_base28[6][25] = {
    {0.85009765625, 1.2998046875, 0.5, -0.2998046875, -0.35009765625, -0.35009765625, -0.2998046875, 0.5, 1.2998046875, 0.85009765625, -0.5, 0, 1.0, 0, -0.5, -0.353553390593274, 0.707106781186548, -0.353553390593274, 0, 0, 0, 0, -0.353553390593274, 0.707106781186548, -0.353553390593274},
    {0.905622728168965, 0, 0, 0, 0, 0, 0, 0, 0, 0.905622728168965, -0.443145751953125, 0.39990234375, 0.60009765625, 0.39990234375, -0.443145751953125, -0.353553390593274, 0.707106781186548, -0.353553390593274, 0, 0, 0, 0, -0.353553390593274, 0.707106781186548, -0.353553390593274},
    {0.85009765625, 0.64990234375, 0.25, -0.14990234375, -0.35009765625, -0.35009765625, -0.14990234375, 0.25, 0.64990234375, 0.85009765625, -1.0, 0, 1.0, 0, -1.0, -0.707106781186548, 0.707106781186548, -0.353553390593274, 0, 0, 0, 0, -0.353553390593274, 0.707106781186548, -0.707106781186548},
    {0.5, 0, -0.5, -0.919100708749311, 0.211993927562764, 0.375, 0.125, 0, 0.777886512701802, -0.070779731515255, 0.25, 0.25, 0.5, -0.353553390593274, -0.353553390593274, 0.125, 0.375, 0, -0.070779731515255, 0.777886512701803, 0, 0.5, -0.5, 0.211993927562764, -0.919100708749311},
    {0.5, 0, 0, 0, 0, 0.375, 0.125, 0.5, 1.131439903295076, -0.282773659078019, 0.25, 0.25, 1.0, -0.565547318156037, -0.565547318156038, 0.125, 0.375, 0.5, -0.282773659078019, 1.131439903295076, 0, 0.5, 0, 0, 0},
    {0.5, 0, -0.25, -0.459550354374656, 0.105996963781382, 0.75, 0.25, 0, 0.777886512701802, -0.070779731515255, 0.5, 0.5, 0.5, -0.353553390593274, -0.353553390593274, 0.25, 0.75, 0, -0.070779731515255, 0.777886512701803, 0, 0.5, -0.25, 0.105996963781382, -0.459550354374656}};
const double h_base46[4][25] = {
    {1.851562500000001, 2.097656250000000, 0.500000000000000, -1.097656250000000, -1.351562500000000,
     -1.351562500000000, -1.097656250000000, 0.500000000000000, 2.097656250000000, 1.851562500000001,
     1.000000000000000, 0.000000000000000, -2.000000000000000, 0.000000000000000, 1.000000000000000,
     0.353553390593274, -0.618718433538229, 0.353553390593274, -0.088388347648318, 0,
     0, -0.088388347648318, 0.353553390593274, -0.618718433538229, 0.353553390593274},
    {2.102851867675782, 0, 0, 0, 0, 0, 0, 0, 0, 2.102851867675782, 0.683105468750000, -0.199707031250000,
     -0.400390625000000, -0.199707031250000, 0.683105468750000, 0.353553390593274, -0.441941738241592,
     0.353553390593274, -0.088388347648318, 0, 0, -0.088388347648318, 0.353553390593274, -0.441941738241592,
     0.353553390593274},
    {0.343750000000000, 0.156250000000000, 0.250000000000000, 0.918410174783309, -0.211303393596761,
     0.312500000000000, 0.187500000000000, 0, -0.919791242715314, 0.212684461528766,
     0.250000000000000, 0.250000000000000, -0.250000000000000, 0.353553390593274, 0.353553390593274,
     0.187500000000000, 0.312500000000000, 0, 0.212684461528766, -0.919791242715314,
     0.156250000000000, 0.343750000000000, 0.250000000000000, -0.211303393596761, 0.918410174783309},
    {0.281250000000000, 0, 0, 0, 0, 0.312500000000000, 0.125000000000000, -1.000000000000000,
     -1.980451414495135, 0.847975710251055, 0.234375000000000, 0.234375000000000, -1.500000000000000,
     0.564856784190035, 0.564856784190035, 0.125000000000000, 0.312500000000000, -1.000000000000000,
     0.847975710251055, -1.980451414495135, 0, 0.281250000000000, 0, 0, 0}};

// forward reflection of pair k at a level of even length L (+ext): cuWT_CDF3_5_{n,d} / cuWT_CDF4_4_{n,d}
template <int WAV>
__device__ __forceinline__ void fwd_reflect(int k, int L, int bcd, int& ai, int& di, float& sa, float& sd) {
    int a = 2 * k, d = 2 * k + 1;
    float s_a = 1.f, s_d = 1.f;
    if (q3_rules(WAV)) {
        if (a < 0) { a = -1 - a; if (bcd) s_a = -1.f; }
        else if (a >= L) { a = 2 * L - 1 - a; if (bcd) s_a = -1.f; }
        if (d < 0) { d = -1 - d; if (bcd) s_d = -1.f; }
        else if (d >= L) { d = 2 * L - 1 - d; if (bcd) s_d = -1.f; }
    } else if (l2_rules(WAV) && bcd == 1) {
        // cuWT_CDF2_6_d (cuWaveletCompute.cuh:271-294): a reflected without a sign, d with one
        if (a < 0) a = -a;
        else if (a > L) a = 2 * L - a;
        if (d < 0) { d = -d; s_d = -1.f; }
        else if (d >= L) { d = 2 * L - d; s_d = -1.f; }
    } else if (l2_rules(WAV)) {
        // cuWT_CDF2_6_n (:255-269) and _z (:296-311, the boundary samples count twice)
        if (a < 0) { a = -a; d = -d; }
        else if (a >= L) { a = 2 * L - a; d = 2 * L - d; }
        if (bcd == 2 && (a == 0 || a == L)) s_a = 2.f;
    } else {
        const int a0 = a;
        if (a < 0) { a = -a; d = -d; if (bcd) { s_a = -1.f; s_d = -1.f; } }
        else if (a >= L) { a = 2 * L - a; d = 2 * L - d; if (bcd) { s_a = -1.f; s_d = -1.f; } }
        if (bcd && a0 == L) s_a = 1.f;
    }
    ai = a; di = d; sa = s_a; sd = s_d;
}

// inverse reflection of index k (a has L+ext entries, d has L): cuWT_CDF3_5_{n,d}_i / cuWT_CDF4_4_{n,d}_i
template <int WAV>
__device__ __forceinline__ void inv_reflect(int k, int L, int bcd, int& ai, int& di, float& sa, float& sd) {
    int a = k, d = k;
    float s_a = 1.f, s_d = 1.f;
    if (q3_rules(WAV)) {
        if (a < 0) { a = -1 - a; if (bcd) s_a = -1.f; else s_d = -1.f; }
        else if (a >= L) { a = 2 * L - 1 - a; if (bcd) s_a = -1.f; else s_d = -1.f; }
        d = a;
    } else if (l2_rules(WAV) && bcd == 1) {
        // cuWT_CDF2_6_d_i (cuWaveletCompute.cuh:668-683)
        if (a < 0) { a = -a; d = -d - 1; s_d = -1.f; }
        else if (a >= L) { a = 2 * L - a; d = 2 * L - d - 1; s_d = -1.f; }
    } else if (bcd != 1) {
        // 'n' (and CDF2.x's 'z', cuWT_CDF2_6_z_i :684-699, sign 2 at the two boundary indices)
        if (bcd == 2 && (a == 0 || a == L)) s_a = 2.f;
        if (a < 0) { a = -a; d = -d - 1; }
        else if (a >= L) { a = 2 * L - a; d = 2 * L - d - 1; }
    } else {
        if (a < 0) { a = -a; d = -d - 1; s_d = -1.f; s_a = -1.f; }
        else if (a >= L) { d = 2 * L - d - 1; s_d = -1.f; }
        if (a > L) { a = 2 * L - a; s_a = -1.f; }
    }
    ai = a; di = d; sa = s_a; sd = s_d;
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

struct TileGeom {
    long s_in;    // stride between consecutive lines of a tile
    long s_out;   // stride of the outer line index
    long pstride; // stride along the transform axis
    int ni;       // lines along the inner index
    int contiguous; // 1: lines are contiguous (y axis)
};

// Reflection tables: for every level, the (index, sign) of each pair a boundary window reads,
// k = -4 .. nch CH + 3 (entry k + 4), computed once per CTA; a boundary window then costs one table
// read per tap instead of the reflection rules.  Entries per level: nch CH + 8.
__host__ __device__ inline int rt_level_entries(int M, int ch) { return (M + ch - 1) / ch * ch + 8; }
__host__ __device__ inline int rt_entries(int N, int levels, bool fwd, int ch) {
    const int ext = N & 1;
    int e = 0;
    for (int l = 2; l < levels; ++l) e += rt_level_entries(fwd ? (1 << l) + ext : (1 << l) + ext, ch);
    return e;
}
__host__ __device__ inline size_t rt_offset(size_t buf_bytes) { return (buf_bytes + 15) / 16 * 16; }

// base-level matrix (nb = 4 or 5) on one column: in[i * pitch] -> out[i * pitch], unrolled so that
// the coefficients stay in registers
template <typename T, int NB>
__device__ __forceinline__ void base_level_n(const double* mat, const T* in, T* out, int pitch) {
    T a[NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) a[i] = in[i * pitch];
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        T s = T(0);
#pragma unroll
        for (int j = 0; j < NB; ++j) s += T(mat[i * NB + j]) * a[j];
        out[i * pitch] = s;
    }
}
template <typename T>
__device__ __forceinline__ void base_level(const double* mat, int nb, const T* in, T* out, int pitch) {
    if (nb == 5) base_level_n<T, 5>(mat, in, out, pitch);
    else base_level_n<T, 4>(mat, in, out, pitch);
}

template <int WAV, bool FWD, typename T, int C>
__global__ void __launch_bounds__(NT) dwt_tile_kernel(const T* __restrict__ src, T* __restrict__ dst, int N,
                                                      int levels, int bcd, TileGeom g) {
    constexpr int CH = ch_of(WAV);
    constexpr int WIN = CH + 8;  // register window (4-pair halo on each side)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    constexpr int CP = C + 1;
    const int tid = threadIdx.x;
    const int ext = N & 1;
    const int i0 = blockIdx.x * C;
    const long obase = (long)blockIdx.y * g.s_out;
    // the three staging buffers, addressed arithmetically (an array of pointers indexed by a run-time
    // buffer number would live in local memory)
    const size_t bstride = (size_t)N * CP;
    auto buf = [sm, bstride](int i) { return sm + (size_t)i * bstride; };

    // ---- reflection tables of every level (see rt_entries), ascending level order
    int4* rt = reinterpret_cast<int4*>(smem_raw + rt_offset((size_t)(FWD ? 2 : 3) * N * CP * sizeof(T)));
    {
        int off = 0;
        for (int l = 2; l < levels; ++l) {
            const int ne = rt_level_entries((1 << l) + ext, CH);
            const int L = FWD ? (1 << (l + 1)) : (1 << l);
            for (int e = tid; e < ne; e += NT) {
                int ai, di;
                float sa, sd;
                if (FWD) {
                    fwd_reflect<WAV>(e - 4, L, bcd, ai, di, sa, sd);
                    ai = clampi(ai, 0, L + ext - 1);
                    di = clampi(di, 0, L + ext - 1);
                } else {
                    inv_reflect<WAV>(e - 4, L, bcd, ai, di, sa, sd);
                    ai = clampi(ai, 0, L + ext - 1);
                    di = clampi(di, 0, L - 1);
                }
                rt[off + e] = make_int4(ai, di, __float_as_int(sa), __float_as_int(sd));
            }
            off += ne;
        }
    }

    // ---- load the tile: C lines of N samples, LU independent loads in flight per thread (a loop
    // of single loads, each waited for before the next, left the pass latency bound)
    constexpr int LU = 8;
    if (g.contiguous) {
        // one warp per line: coalesced along the line, no index division
        for (int col = tid >> 5; col < C; col += NT / 32) {
            const bool ok = i0 + col < g.ni;
            const T* line = src + obase + (long)(ok ? i0 + col : 0) * g.s_in;
            for (int p0 = tid & 31; p0 < N; p0 += 32 * LU) {
                T v[LU];
#pragma unroll
                for (int u = 0; u < LU; ++u) {
                    const int p = p0 + 32 * u;
                    v[u] = (ok && p < N) ? line[p] : T(0);
                }
#pragma unroll
                for (int u = 0; u < LU; ++u) {
                    const int p = p0 + 32 * u;
                    if (p < N) buf(0)[p * CP + col] = v[u];
                }
            }
        }
    } else {
        // NT is a multiple of C: a thread keeps its column, positions advance by NT / C
        const int col = tid % C;
        const bool ok = i0 + col < g.ni;
        const T* cs = src + obase + (long)(ok ? i0 + col : 0) * g.s_in;
        constexpr int PS = NT / C;
        for (int p0 = tid / C; p0 < N; p0 += PS * LU) {
            T v[LU];
#pragma unroll
            for (int u = 0; u < LU; ++u) {
                const int p = p0 + PS * u;
                v[u] = (ok && p < N) ? cs[(long)p * g.pstride] : T(0);
            }
#pragma unroll
            for (int u = 0; u < LU; ++u) {
                const int p = p0 + PS * u;
                if (p < N) buf(0)[p * CP + col] = v[u];
            }
        }
    }
    __syncthreads();

    const int nb = 4 + ext;
    int outbuf;
    if (FWD) {
        int cur = 0;
        int rt_off = 0;
        for (int l = 2; l < levels; ++l) rt_off += rt_level_entries((1 << l) + ext, CH);
        for (int l = levels - 1; l >= 2; --l) {
            rt_off -= rt_level_entries((1 << l) + ext, CH);
            const int4* tb = rt + rt_off;
            const int L = 1 << (l + 1);
            const int M = (L >> 1) + ext;
            const int nd = L >> 1;
            const T* S = buf(cur);
            T* D = buf(cur ^ 1);
            const int nch = (M + CH - 1) / CH;
            for (int t = tid; t < C * nch; t += NT) {
                const int col = t % C, k0 = (t / C) * CH;
                T A[WIN], Dd[WIN];
                // CDF2.x: the detail's reflection sign applies after the predict and the approximation's
                // is divided out at the end (cuUpdateCdf26_ad), so they are kept apart from the values
                T SAw[WIN], SDw[WIN];
                if (k0 >= 4 + (bcd == 2) && 2 * (k0 + WIN - 4) <= L) {
                    // interior window: no reflection (CDF2.x 'z' weighs the boundary samples twice)
                    const T* base = S + (2 * (k0 - 4)) * CP + col;
#pragma unroll
                    for (int w = 0; w < WIN; ++w) {
                        A[w] = base[(2 * w) * CP];
                        Dd[w] = base[(2 * w + 1) * CP];
                        SAw[w] = T(1);
                        SDw[w] = T(1);
                    }
                } else {
#pragma unroll
                    for (int w = 0; w < WIN; ++w) {
                        const int4 e = tb[k0 + w];
                        A[w] = (WAV == WP_ID_CDF2_0 ? T(1) : T(__int_as_float(e.z))) * S[e.x * CP + col];
                        if (l2_rules(WAV)) {
                            Dd[w] = S[e.y * CP + col];
                            SAw[w] = T(__int_as_float(e.z));
                            SDw[w] = T(__int_as_float(e.w));
                        } else {
                            Dd[w] = T(__int_as_float(e.w)) * S[e.y * CP + col];
                        }
                    }
                }
                if (WAV == WP_ID_CDF2_0) {
                    // cuUpdateCdf20_ad: the predict on the samples as read (no sign: at an output pair
                    // both neighbours lie inside the line), the detail's scale negated
#pragma unroll
                    for (int j = 0; j < CH; ++j) {
                        const int w = j + 4, k = k0 + j;
                        const T dv = Dd[w] + (T(K2<WP_ID_CDF2_6>::fp0) * A[w] + T(K2<WP_ID_CDF2_6>::fp1) * A[w + 1]);
                        if (k < M) D[k * CP + col] = A[w] * T(K2<WP_ID_CDF2_6>::scl0);
                        if (k < nd) D[(M + k) * CP + col] = dv * T(-K2<WP_ID_CDF2_6>::scl1);
                    }
                } else if (is_t1(WAV)) {
                    // cuUpdateCdf11_ad / cuUpdateCdf17_ad (signs applied at the load)
#pragma unroll
                    for (int w = 0; w < WIN; ++w) Dd[w] = Dd[w] + T(KT::fp) * A[w];
#pragma unroll
                    for (int j = 0; j < CH; ++j) {
                        const int w = j + 4, k = k0 + j;
                        T s = A[w];
                        if (WAV == WP_ID_CDF1_1) {
                            s += T(KT::fu) * Dd[w];
                        } else {
#pragma unroll
                            for (int i = 6; i >= 0; --i) s += T(KT::t7(i)) * Dd[w + 3 - i];
                        }
                        if (k < M) D[k * CP + col] = s * T(KT::scl0);
                        if (k < nd) D[(M + k) * CP + col] = Dd[w] * T(WAV == WP_ID_CDF1_1 ? KT::scl1 : KT::scl7_1);
                    }
                } else if (is_l2(WAV)) {
                    constexpr int NTP = K2<WAV>::NTAP, LO = NTP / 2;
#pragma unroll
                    for (int w = 0; w < WIN - 1; ++w)
                        Dd[w] = (Dd[w] + T(K2<WAV>::fp0) * A[w] + T(K2<WAV>::fp1) * A[w + 1]) * SDw[w];
#pragma unroll
                    for (int j = 0; j < CH; ++j) {
                        const int w = j + 4;
                        T s = A[w];
#pragma unroll
                        for (int t = 0; t < NTP; ++t) s = s + T(K2<WAV>::u(NTP - 1 - t)) * Dd[w - LO + t];
                        const int k = k0 + j;
                        if (k < M) D[k * CP + col] = s * T(K2<WAV>::scl0) / SAw[w];
                        if (k < nd) D[(M + k) * CP + col] = Dd[w] * T(K2<WAV>::scl1);
                    }
                } else if (is_q3(WAV)) {
#pragma unroll
                    for (int w = WIN - 1; w >= 1; --w) A[w] = A[w] + T(K37::fu1) * Dd[w - 1];
#pragma unroll
                    for (int w = 1; w < WIN - 1; ++w) Dd[w] = Dd[w] + T(K37::fp0) * A[w + 1] + T(K37::fp1) * A[w];
#pragma unroll
                    for (int j = 0; j < CH; ++j) {
                        const int w = j + 4;
                        T s = A[w] + T(K3<WAV>::q6) * Dd[w - 3] + T(K3<WAV>::q5) * Dd[w - 2] + T(K3<WAV>::q4) * Dd[w - 1] +
                              T(K3<WAV>::q3) * Dd[w] + T(K3<WAV>::q2) * Dd[w + 1] + T(K3<WAV>::q1) * Dd[w + 2] +
                              T(K3<WAV>::q0) * Dd[w + 3];
                        const int k = k0 + j;
                        if (k < M) D[k * CP + col] = s * T(K37::scl0);
                        if (k < nd) D[(M + k) * CP + col] = Dd[w] * T(K37::scl1);
                    }
                } else {
#pragma unroll
                    for (int w = WIN - 1; w >= 1; --w)
                        A[w] = A[w] + T(K46::fu1_1) * Dd[w - 1] + T(K46::fu1_0) * Dd[w];
#pragma unroll
                    for (int w = 1; w < WIN - 1; ++w) Dd[w] = Dd[w] + T(K46::fp1) * A[w] + T(K46::fp0) * A[w + 1];
#pragma unroll
                    for (int j = 0; j < CH; ++j) {
                        const int w = j + 4;
                        T s = WAV == WP_ID_CDF4_4
                                  ? A[w] + T(K44::d3) * Dd[w - 2] + T(K44::d2) * Dd[w - 1] + T(K44::d1) * Dd[w] +
                                        T(K44::d0) * Dd[w + 1]
                                  : A[w] + T(K46::c5) * Dd[w - 3] + T(K46::c4) * Dd[w - 2] + T(K46::c3) * Dd[w - 1] +
                                        T(K46::c2) * Dd[w] + T(K46::c1) * Dd[w + 1] + T(K46::c0) * Dd[w + 2];
                        const int k = k0 + j;
                        if (k < M) D[k * CP + col] = s * T(K46::scl0);
                        if (k < nd) D[(M + k) * CP + col] = Dd[w] * T(K46::scl1);
                    }
                }
            }
            __syncthreads();
            cur ^= 1;
        }
        // base level: nb x nb matrix on the remaining approximation coefficients
        const double* mat = WAV == WP_ID_CDF3_7   ? c_base37[bcd]
                            : WAV == WP_ID_CDF2_0 ? c_base20[0]
                            : WAV == WP_ID_CDF1_1 ? c_base11[0]
                            : WAV == WP_ID_CDF1_7 ? c_base17[bcd]
                            : WAV == WP_ID_CDF3_5 ? c_base35[bcd]
                            : WAV == WP_ID_CDF4_4 ? c_base44[bcd]
                            : WAV == WP_ID_CDF2_6 ? c_base26[bcd]
                            : WAV == WP_ID_CDF2_8 ? c_base28[bcd]
                                                  : c_base46[bcd];
        if (tid < C) base_level<T>(mat, nb, buf(cur) + tid, buf(cur ^ 1) + tid, CP);
        __syncthreads();
        outbuf = -1;  // position dependent, resolved below
    } else {
        const double* mat = WAV == WP_ID_CDF3_7   ? c_base37[2 + bcd]
                            : WAV == WP_ID_CDF2_0 ? c_base20[1]
                            : WAV == WP_ID_CDF1_1 ? c_base11[1]
                            : WAV == WP_ID_CDF1_7 ? c_base17[2 + bcd]
                            : WAV == WP_ID_CDF3_5 ? c_base35[2 + bcd]
                            : WAV == WP_ID_CDF4_4 ? c_base44[2 + bcd]
                            : WAV == WP_ID_CDF2_6 ? c_base26[3 + bcd]
                            : WAV == WP_ID_CDF2_8 ? c_base28[3 + bcd]
                                                  : c_base46[2 + bcd];
        if (tid < C) base_level<T>(mat, nb, buf(0) + tid, buf(1) + tid, CP);
        __syncthreads();
        int cur = 1;
        int rt_off = 0;
        for (int l = 2; l < levels; ++l) {
            const int4* tb = rt + rt_off;
            rt_off += rt_level_entries((1 << l) + ext, CH);
            const int L = 1 << l;
            const int NA = L + ext;
            const T* Sa = buf(cur);
            const T* Sd = buf(0) + (size_t)NA * CP;
            T* D = buf(3 - cur);
            const int nch = (NA + CH - 1) / CH;
            for (int t = tid; t < C * nch; t += NT) {
                const int col = t % C, k0 = (t / C) * CH;
                T A[WIN], Dd[WIN], SA[WIN], SD[WIN];
                if (k0 >= 4 + (bcd == 2) && k0 + WIN - 4 <= L) {
                    // interior window: no reflection
#pragma unroll
                    for (int w = 0; w < WIN; ++w) {
                        A[w] = Sa[(k0 - 4 + w) * CP + col];
                        Dd[w] = Sd[(k0 - 4 + w) * CP + col];
                        SA[w] = T(1);
                        SD[w] = T(1);
                    }
                } else {
#pragma unroll
                    for (int w = 0; w < WIN; ++w) {
                        const int4 e = tb[k0 + w];
                        A[w] = Sa[e.x * CP + col];
                        Dd[w] = Sd[e.y * CP + col];
                        SA[w] = T(__int_as_float(e.z));
                        SD[w] = T(__int_as_float(e.w));
                    }
                }
                if (WAV == WP_ID_CDF2_0) {
                    // cuUpdateCdf20_ad_i
#pragma unroll
                    for (int j = 0; j < CH; ++j) {
                        const int w = j + 4, k = k0 + j;
                        const T a0 = SA[w] * A[w] * T(K2<WP_ID_CDF2_6>::scl1);
                        const T a1 = SA[w + 1] * A[w + 1] * T(K2<WP_ID_CDF2_6>::scl1);
                        const T dv = -SD[w] * Dd[w] * T(K2<WP_ID_CDF2_6>::scl0);
                        if (k < NA) D[(2 * k) * CP + col] = a0;
                        if (k < L)
                            D[(2 * k + 1) * CP + col] =
                                dv - (T(K2<WP_ID_CDF2_6>::fp1) * a0 + T(K2<WP_ID_CDF2_6>::fp0) * a1);
                    }
                } else if (WAV == WP_ID_CDF1_1) {
                    // cuUpdateCdf11_ad_i (no sign: the step reads no neighbour)
#pragma unroll
                    for (int j = 0; j < CH; ++j) {
                        const int w = j + 4, k = k0 + j;
                        const T dv = Dd[w] * T(KT::scl0);
                        const T av = A[w] * T(KT::scl1) - T(KT::fu) * dv;
                        if (k < NA) D[(2 * k) * CP + col] = av;
                        if (k < L) D[(2 * k + 1) * CP + col] = dv - T(KT::fp) * av;
                    }
                } else if (WAV == WP_ID_CDF1_7) {
                    // cuUpdateCdf17_ad_i: signed and scaled (by division, as the reference), the update
                    // undone, then the predict
#pragma unroll
                    for (int w = 0; w < WIN; ++w) {
                        Dd[w] = SD[w] * Dd[w] / T(KT::scl7_1);
                        A[w] = SA[w] * A[w] / T(KT::scl0);
                    }
#pragma unroll
                    for (int j = 0; j < CH; ++j) {
                        const int w = j + 4, k = k0 + j;
                        T av = A[w];
#pragma unroll
                        for (int i = 6; i >= 0; --i) av -= T(KT::t7(i)) * Dd[w + 3 - i];
                        if (k < NA) D[(2 * k) * CP + col] = av;
                        if (k < L) D[(2 * k + 1) * CP + col] = Dd[w] - T(KT::fp) * av;
                    }
                } else if (is_l2(WAV)) {
                    // cuUpdateCdf26_ad_i / cuUpdateCdf28_ad_i: scale, undo the update, undo the predict,
                    // divide out the approximation's sign
                    constexpr int NTP = K2<WAV>::NTAP, LO = NTP / 2;
#pragma unroll
                    for (int w = 0; w < WIN; ++w) {
                        Dd[w] = SD[w] * Dd[w] * T(K2<WAV>::scl0);
                        A[w] = SA[w] * A[w] * T(K2<WAV>::scl1);
                    }
#pragma unroll
                    for (int w = LO; w <= WIN - LO; ++w) {
                        T t = A[w];
#pragma unroll
                        for (int i = 0; i < NTP; ++i) t = t - T(K2<WAV>::u(NTP - 1 - i)) * Dd[w - LO + i];
                        A[w] = t;
                    }
#pragma unroll
                    for (int j = 0; j < CH; ++j) {
                        const int w = j + 4, k = k0 + j;
                        if (k < NA) D[(2 * k) * CP + col] = A[w] / SA[w];
                        if (k < L)
                            D[(2 * k + 1) * CP + col] = Dd[w] - (T(K2<WAV>::fp1) * A[w] + T(K2<WAV>::fp0) * A[w + 1]);
                    }
                } else if (is_q3(WAV)) {
#pragma unroll
                    for (int w = 0; w < WIN; ++w) {
                        A[w] = SA[w] * A[w] * T(K37::scl1);
                        Dd[w] = SD[w] * Dd[w] * T(K37::scl0);
                    }
#pragma unroll
                    for (int w = 3; w < WIN - 3; ++w)
                        A[w] = A[w] - (T(K3<WAV>::q6) * Dd[w - 3] + T(K3<WAV>::q5) * Dd[w - 2] + T(K3<WAV>::q4) * Dd[w - 1] +
                                       T(K3<WAV>::q3) * Dd[w] + T(K3<WAV>::q2) * Dd[w + 1] + T(K3<WAV>::q1) * Dd[w + 2] +
                                       T(K3<WAV>::q0) * Dd[w + 3]);
#pragma unroll
                    for (int w = 3; w < WIN - 4; ++w) Dd[w] = Dd[w] - (T(K37::fp1) * A[w] + T(K37::fp0) * A[w + 1]);
#pragma unroll
                    for (int j = 0; j < CH; ++j) {
                        const int w = j + 4, k = k0 + j;
                        const T av = A[w] - T(K37::fu1) * Dd[w - 1];
                        if (k < NA) D[(2 * k) * CP + col] = av;
                        if (k < L) D[(2 * k + 1) * CP + col] = Dd[w];
                    }
                } else {
#pragma unroll
                    for (int w = 0; w < WIN; ++w) {
                        Dd[w] = SD[w] * Dd[w] * T(K46::scli1);
                        A[w] = SA[w] * A[w] * T(K46::scli0);
                    }
#pragma unroll
                    for (int w = 3; w < WIN - 2; ++w)
                        A[w] = SA[w] * (A[w] - (WAV == WP_ID_CDF4_4
                                                    ? T(K44::d3) * Dd[w - 2] + T(K44::d2) * Dd[w - 1] +
                                                          T(K44::d1) * Dd[w] + T(K44::d0) * Dd[w + 1]
                                                    : T(K46::c5) * Dd[w - 3] + T(K46::c4) * Dd[w - 2] +
                                                          T(K46::c3) * Dd[w - 1] + T(K46::c2) * Dd[w] +
                                                          T(K46::c1) * Dd[w + 1] + T(K46::c0) * Dd[w + 2]));
#pragma unroll
                    for (int w = 0; w < WIN; ++w) Dd[w] = SD[w] * Dd[w];
#pragma unroll
                    for (int w = 3; w < WIN - 3; ++w)
                        Dd[w] = SD[w] * (Dd[w] - (T(K46::fp1) * A[w] + T(K46::fp0) * A[w + 1]));
#pragma unroll
                    for (int j = 0; j < CH; ++j) {
                        const int w = j + 4, k = k0 + j;
                        const T av = A[w] - (T(K46::fu1_1) * Dd[w - 1] + T(K46::fu1_0) * Dd[w]);
                        if (k < NA) D[(2 * k) * CP + col] = av;
                        if (k < L) D[(2 * k + 1) * CP + col] = Dd[w];
                    }
                }
            }
            __syncthreads();
            cur = 3 - cur;
        }
        outbuf = cur;
    }

    // ---- store the tile.  The forward result's position p lives in one buffer per Mallat region
    // (the base, then detail level l at [2^l + ext, 2^(l+1) + ext)): a thread walks its positions with
    // a running global pointer and shared index and re-selects the buffer only when p enters the next
    // region (the inverse result is all in outbuf).
    const int basebuf = (levels - 1) & 1;
    auto region = [&](int p, int& b, int& next) {
        if (outbuf >= 0) {
            b = outbuf;
            next = N;
        } else if (p < nb) {
            b = basebuf;
            next = nb;
        } else {
            const int lg = 31 - __clz(p - ext);
            b = (levels - lg) & 1;
            next = (2 << lg) + ext;
        }
    };
    if (g.contiguous) {
        for (int col = tid >> 5; col < C; col += NT / 32) {
            if (i0 + col >= g.ni) continue;
            T* line = dst + obase + (long)(i0 + col) * g.s_in;
            int p = tid & 31, b, next;
            region(p, b, next);
            for (; p < N; p += 32) {
                if (p >= next) region(p, b, next);
                line[p] = buf(b)[p * CP + col];
            }
        }
    } else {
        // NT is a multiple of C: a thread keeps its column, positions advance by NT / C
        constexpr int PS = NT / C;
        const int col = tid % C;
        if (i0 + col < g.ni) {
            int p = tid / C, b, next;
            T* gp = dst + obase + (long)(i0 + col) * g.s_in + (long)p * g.pstride;
            const long gstep = (long)PS * g.pstride;
            int si = p * CP + col;
            region(p, b, next);
            for (; p < N; p += PS, gp += gstep, si += PS * CP) {
                if (p >= next) region(p, b, next);
                *gp = buf(b)[si];
            }
        }
    }
}

bool g_const_ready[64] = {false};
std::mutex g_const_mu;

// Uploads the filter tables once per device (synchronous copy: run at handle creation, before any
// stream capture).
cudaError_t ensure_constants() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(g_const_mu);
    if (dev < 64 && g_const_ready[dev]) return cudaSuccess;
    double b37[4][16], b46[4][25];
    memcpy(b37, h_base37, sizeof(b37));
    memcpy(b46, h_base46, sizeof(b46));
    // stored order: forward n, forward d, inverse n, inverse d
    e = cudaMemcpyToSymbol(c_base37, b37, sizeof(b37));
    if (e != cudaSuccess) return e;
    e = cudaMemcpyToSymbol(c_base46, b46, sizeof(b46));
    if (e != cudaSuccess) return e;
    e = cudaMemcpyToSymbol(c_base35, h_base35, sizeof(h_base35));
    if (e != cudaSuccess) return e;
    e = cudaMemcpyToSymbol(c_base44, h_base44, sizeof(h_base44));
    if (e != cudaSuccess) return e;
    e = cudaMemcpyToSymbol(c_base26, h_base26, sizeof(h_base26));
    if (e != cudaSuccess) return e;
    e = cudaMemcpyToSymbol(c_base28, h_base28, sizeof(h_base28));
    if (e != cudaSuccess) return e;
    e = cudaMemcpyToSymbol(c_base20, h_base20, sizeof(h_base20));
    if (e != cudaSuccess) return e;
    e = cudaMemcpyToSymbol(c_base11, h_base11, sizeof(h_base11));
    if (e != cudaSuccess) return e;
    e = cudaMemcpyToSymbol(c_base17, h_base17, sizeof(h_base17));
    if (e != cudaSuccess) return e;
    if (dev < 64) g_const_ready[dev] = true;
    return cudaSuccess;
}

template <typename T>
size_t dwt_smem(int N, int levels, bool fwd, int C, int ch) {
    return rt_offset((size_t)(fwd ? 2 : 3) * N * (C + 1) * sizeof(T)) + 16 * (size_t)rt_entries(N, levels, fwd, ch);
}

template <int WAV, bool FWD, typename T, int C>
cudaError_t launch_one(const T* src, T* dst, int N, int levels, int bcd, TileGeom g, int nouter, cudaStream_t s) {
    const size_t smem = dwt_smem<T>(N, levels, FWD, C, ch_of(WAV));
    auto kern = dwt_tile_kernel<WAV, FWD, T, C>;
    cudaError_t e = wp_set_smem(kern, smem);
    if (e != cudaSuccess) return e;
    dim3 grid((g.ni + C - 1) / C, nouter);
    const int tok = wp_prof_start(s);
    kern<<<grid, NT, smem, s>>>(src, dst, N, levels, bcd, g);
    e = cudaGetLastError();
    // algorithmic bytes: every element of the transformed array read once and written once
    wp_prof_stop(tok, FWD ? "dwt_forward" : "dwt_inverse", 2.0 * sizeof(T) * N * (double)g.ni * nouter, s);
    return e;
}

// Tile widths chosen by the autotuner, per (device, wavelet, direction, precision, line length,
// lines, outer extent, axis kind); a width changes only the grid, never a result.
std::mutex g_c_mu;
std::map<std::tuple<int, int, int, int, int, int, int, int>, int> g_c_cache;

std::tuple<int, int, int, int, int, int, int, int> c_key(int wav, bool fwd, int tsize, int N, const TileGeom& g,
                                                         int nouter) {
    int dev = 0;
    cudaGetDevice(&dev);
    return std::make_tuple(dev, wav, fwd ? 1 : 0, tsize, N, g.ni, nouter, g.contiguous);
}

// -1: let launch_c decide (cache, then heuristic); otherwise force this tile width
thread_local int t_force_c = -1;

template <int WAV, bool FWD, typename T>
cudaError_t launch_c(const T* src, T* dst, int N, int levels, int bcd, TileGeom g, int nouter, cudaStream_t s) {
    // widest tile whose staging fits ~100 KB (two CTAs per SM) while keeping >= 2 CTAs per SM busy,
    // unless the autotuner measured another width for this shape
    int C = 32;
    const long sms = wp_sm_count();
    while (C > 4) {
        const size_t smem = dwt_smem<T>(N, levels, FWD, C, ch_of(WAV));
        const long ctas = (long)((g.ni + C - 1) / C) * nouter;
        if (smem <= 100 * 1024 && ctas >= 2 * sms) break;
        C >>= 1;
    }
    if (t_force_c > 0) {
        C = t_force_c;
    } else {
        std::lock_guard<std::mutex> lk(g_c_mu);
        auto it = g_c_cache.find(c_key(WAV, FWD, (int)sizeof(T), N, g, nouter));
        if (it != g_c_cache.end()) C = it->second;
    }
    const size_t smem = dwt_smem<T>(N, levels, FWD, C, ch_of(WAV));
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    switch (C) {
        case 32: return launch_one<WAV, FWD, T, 32>(src, dst, N, levels, bcd, g, nouter, s);
        case 16: return launch_one<WAV, FWD, T, 16>(src, dst, N, levels, bcd, g, nouter, s);
        case 8: return launch_one<WAV, FWD, T, 8>(src, dst, N, levels, bcd, g, nouter, s);
        default: return launch_one<WAV, FWD, T, 4>(src, dst, N, levels, bcd, g, nouter, s);
    }
}

}  // namespace

template <typename T>
wp_status wp_dwt_axis_launch(T* dst, const T* src, int DX, int DY, int DZ, int levels, char axis, int wavelet,
                             char bc, int forward, cudaStream_t stream) {
    if (!dst || DX <= 0 || DY <= 0 || DZ <= 0) { wp_set_error_msg("wp_dwt1d: bad arguments"); return WP_ERR_INVALID_ARG; }
    if (!src) src = dst;
    const bool shortf = wavelet == WP_ID_CDF2_0 || is_t1(wavelet);
    if (!is_q3(wavelet) && !is_c4(wavelet) && !is_l2(wavelet) && !shortf) {
        wp_set_error_msg("wp_dwt1d: wavelet must be CDF3.5, CDF3.7, CDF4.4, CDF4.6, CDF2.6, CDF2.8, CDF2.0, "
                         "CDF1.1 or CDF1.7");
        return WP_ERR_UNSUPPORTED;
    }
    // the short families register 'n' and 'd' only (cuWHHDForward.cu:998-1080)
    if (shortf && bc != 'n' && bc != 'd') {
        wp_set_error_msg("wp_dwt1d: CDF2.0, CDF1.1 and CDF1.7 take bc 'n' or 'd'");
        return WP_ERR_INVALID_ARG;
    }
    // 'z': CDF3.x treat it as 'd', CDF4.x as 'n' (cuWHHDForward.cu:760-765, 843-848, 886-891, 970-975);
    // CDF2.x have a rule of their own (:802-828, 928-933)
    if (bc == 'z' && !is_l2(wavelet)) bc = is_q3(wavelet) ? 'd' : 'n';
    if (bc != 'n' && bc != 'd' && bc != 'z') { wp_set_error_msg("wp_dwt1d: bc must be 'n', 'd' or 'z'"); return WP_ERR_INVALID_ARG; }
    TileGeom g;
    int N, nouter;
    switch (axis) {
        case 'y': case 'Y': N = DY; g.s_in = DY; g.ni = DX; g.s_out = (long)DX * DY; nouter = DZ; g.pstride = 1; g.contiguous = 1; break;
        case 'x': case 'X': N = DX; g.s_in = 1; g.ni = DY; g.s_out = (long)DX * DY; nouter = DZ; g.pstride = DY; g.contiguous = 0; break;
        case 'z': case 'Z': N = DZ; g.s_in = 1; g.ni = DY; g.s_out = DY; nouter = DX; g.pstride = (long)DX * DY; g.contiguous = 0; break;
        default: wp_set_error_msg("wp_dwt1d: direction must be x, y or z"); return WP_ERR_INVALID_ARG;
    }
    const int ext = N & 1;
    if (levels < 2 || levels > 12 || (1 << levels) != N - ext) {
        wp_set_error_msg("wp_dwt1d: line length must be 2^levels (+1), levels in [2, 12]");
        return WP_ERR_INVALID_ARG;
    }
    if (nouter > 65535) { wp_set_error_msg("wp_dwt1d: outer extent too large"); return WP_ERR_UNSUPPORTED; }
    WP_CUDA_TRY(ensure_constants());
    if ((wavelet == WP_ID_CDF4_4 || l2_rules(wavelet)) && !(N & 1)) {
        // their base matrices act on five coefficients: whole-sample lines of 2^levels + 1
        wp_set_error_msg("wp_dwt1d: CDF4.4 and CDF2.x lines have 2^levels + 1 samples");
        return WP_ERR_INVALID_ARG;
    }
    if (is_t1(wavelet) && (N & 1)) {
        // their base matrices act on four coefficients
        wp_set_error_msg("wp_dwt1d: CDF1.x lines have 2^levels samples");
        return WP_ERR_INVALID_ARG;
    }
    const int bcd = bc == 'd' ? 1 : (bc == 'z' ? 2 : 0);
    cudaError_t e;
    if (wavelet == WP_ID_CDF3_7)
        e = forward ? launch_c<WP_ID_CDF3_7, true, T>(src, dst, N, levels, bcd, g, nouter, stream)
                    : launch_c<WP_ID_CDF3_7, false, T>(src, dst, N, levels, bcd, g, nouter, stream);
    else if (wavelet == WP_ID_CDF3_5)
        e = forward ? launch_c<WP_ID_CDF3_5, true, T>(src, dst, N, levels, bcd, g, nouter, stream)
                    : launch_c<WP_ID_CDF3_5, false, T>(src, dst, N, levels, bcd, g, nouter, stream);
    else if (wavelet == WP_ID_CDF4_4)
        e = forward ? launch_c<WP_ID_CDF4_4, true, T>(src, dst, N, levels, bcd, g, nouter, stream)
                    : launch_c<WP_ID_CDF4_4, false, T>(src, dst, N, levels, bcd, g, nouter, stream);
    else if (wavelet == WP_ID_CDF2_6)
        e = forward ? launch_c<WP_ID_CDF2_6, true, T>(src, dst, N, levels, bcd, g, nouter, stream)
                    : launch_c<WP_ID_CDF2_6, false, T>(src, dst, N, levels, bcd, g, nouter, stream);
    else if (wavelet == WP_ID_CDF2_8)
        e = forward ? launch_c<WP_ID_CDF2_8, true, T>(src, dst, N, levels, bcd, g, nouter, stream)
                    : launch_c<WP_ID_CDF2_8, false, T>(src, dst, N, levels, bcd, g, nouter, stream);
    else if (wavelet == WP_ID_CDF2_0)
        e = forward ? launch_c<WP_ID_CDF2_0, true, T>(src, dst, N, levels, bcd, g, nouter, stream)
                    : launch_c<WP_ID_CDF2_0, false, T>(src, dst, N, levels, bcd, g, nouter, stream);
    else if (wavelet == WP_ID_CDF1_1)
        e = forward ? launch_c<WP_ID_CDF1_1, true, T>(src, dst, N, levels, bcd, g, nouter, stream)
                    : launch_c<WP_ID_CDF1_1, false, T>(src, dst, N, levels, bcd, g, nouter, stream);
    else if (wavelet == WP_ID_CDF1_7)
        e = forward ? launch_c<WP_ID_CDF1_7, true, T>(src, dst, N, levels, bcd, g, nouter, stream)
                    : launch_c<WP_ID_CDF1_7, false, T>(src, dst, N, levels, bcd, g, nouter, stream);
    else
        e = forward ? launch_c<WP_ID_CDF4_6, true, T>(src, dst, N, levels, bcd, g, nouter, stream)
                    : launch_c<WP_ID_CDF4_6, false, T>(src, dst, N, levels, bcd, g, nouter, stream);
    if (e != cudaSuccess) { wp_set_cuda_error(e, "dwt launch", __FILE__, __LINE__); return WP_ERR_CUDA; }
    return WP_OK;
}

// Times the pass over the tile widths 4..32 that fit shared memory (median of three single launches,
// in place on buf) and records the fastest for this shape.  Synchronous; buf's contents are
// overwritten.
template <typename T>
wp_status wp_dwt_axis_tune(T* buf, int DX, int DY, int DZ, int levels, char axis, int wavelet, char bc, int forward,
                           cudaStream_t s) {
    const int N = (axis == 'y' || axis == 'Y') ? DY : (axis == 'x' || axis == 'X') ? DX : DZ;
    cudaEvent_t a, b;
    WP_CUDA_TRY(cudaEventCreate(&a));
    WP_CUDA_TRY(cudaEventCreate(&b));
    float best = 1e30f;
    int best_c = -1;
    wp_status st = WP_OK;
    for (int C = 4; C <= 32 && st == WP_OK; C *= 2) {
        if (dwt_smem<T>(N, levels, forward != 0, C, ch_of(wavelet)) > 227 * 1024) break;
        t_force_c = C;
        std::vector<float> t;
        for (int r = 0; r < 4 && st == WP_OK; ++r) {
            cudaEventRecord(a, s);
            st = wp_dwt_axis_launch<T>(buf, buf, DX, DY, DZ, levels, axis, wavelet, bc, forward, s);
            cudaEventRecord(b, s);
            cudaEventSynchronize(b);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            if (r > 0) t.push_back(ms);
        }
        t_force_c = -1;
        if (st != WP_OK) break;
        std::sort(t.begin(), t.end());
        if (t[1] < best) {
            best = t[1];
            best_c = C;
        }
    }
    t_force_c = -1;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (st != WP_OK || best_c < 0) return st;
    TileGeom g;
    int nouter;
    switch (axis) {
        case 'y': case 'Y': g.ni = DX; nouter = DZ; g.contiguous = 1; break;
        case 'x': case 'X': g.ni = DY; nouter = DZ; g.contiguous = 0; break;
        default: g.ni = DY; nouter = DX; g.contiguous = 0; break;
    }
    const int wav = wavelet;
    std::lock_guard<std::mutex> lk(g_c_mu);
    g_c_cache[c_key(wav, forward != 0, (int)sizeof(T), N, g, nouter)] = best_c;
    return WP_OK;
}
template wp_status wp_dwt_axis_tune<float>(float*, int, int, int, int, char, int, char, int, cudaStream_t);

template wp_status wp_dwt_axis_launch<float>(float*, const float*, int, int, int, int, char, int, char, int, cudaStream_t);
template wp_status wp_dwt_axis_launch<double>(double*, const double*, int, int, int, int, char, int, char, int,
                                              cudaStream_t);

cudaError_t wp_dwt_prepare() { return ensure_constants(); }

extern "C" CUWHHD_API wp_status wp_dwt1d(float* dst, const float* src, int dim_x, int dim_y, int dim_z, int levels,
                                         char direction, char bc, int wavelet, int forward, void* stream) {
    return wp_dwt_axis_launch<float>(dst, src, dim_x, dim_y, dim_z, levels, direction, wavelet, bc, forward,
                                     (cudaStream_t)stream);
}

extern "C" CUWHHD_API wp_status wp_dwt1d_f64(double* dst, const double* src, int dim_x, int dim_y, int dim_z,
                                             int levels, char direction, char bc, int wavelet, int forward,
                                             void* stream) {
    return wp_dwt_axis_launch<double>(dst, src, dim_x, dim_y, dim_z, levels, direction, wavelet, bc, forward,
                                      (cudaStream_t)stream);
}

// ---- inner-product diagonal: inverse-transform the identity in FP64, sum squares per row
namespace {
__global__ void eye_kernel(double* m, int dim) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long n = (long)dim * dim;
    if (i < n) m[i] = (i / dim == i % dim) ? 1.0 : 0.0;
}
__global__ void row_sumsq_kernel(const double* m, double* out, int dim) {
    int row = blockIdx.x;
    double s = 0.0;
    for (int j = threadIdx.x; j < dim; j += blockDim.x) {
        double v = m[(long)row * dim + j];
        s += v * v;
    }
    __shared__ double red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[row] = red[0];
}
}  // namespace

wp_status wp_ip_diag_device(double* d_out, int dim, int wavelet, char bc, cudaStream_t s) {
    int levels = 0;
    while ((2 << levels) <= dim) ++levels;
    double* m = nullptr;
    WP_CUDA_TRY(cudaMallocAsync((void**)&m, sizeof(double) * (size_t)dim * dim, s));
    {
        const int tok = wp_prof_start(s);
        eye_kernel<<<wp_cdiv((size_t)dim * dim, 256), 256, 0, s>>>(m, dim);
        wp_prof_stop(tok, "ip_identity", 8.0 * dim * dim, s);
    }
    wp_status st = wp_dwt_axis_launch<double>(m, m, dim, dim, 1, levels, 'y', wavelet, bc, 0, s);
    if (st == WP_OK) {
        const int tok = wp_prof_start(s);
        row_sumsq_kernel<<<dim, 256, 0, s>>>(m, d_out, dim);
        cudaError_t e = cudaGetLastError();
        wp_prof_stop(tok, "ip_rowsumsq", 8.0 * dim * dim, s);
        if (e != cudaSuccess) { wp_set_cuda_error(e, "row_sumsq", __FILE__, __LINE__); st = WP_ERR_CUDA; }
    }
    cudaFreeAsync(m, s);
    return st;
}

namespace {
__global__ void unit_pair_kernel(double* m, int dim) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 2 * dim) m[i] = (i == 0 || i == dim + 1) ? 1.0 : 0.0;
}
__global__ void dot_pair_kernel(const double* m, double* out, int dim) {
    double s = 0.0;
    for (int j = threadIdx.x; j < dim; j += blockDim.x) s += m[j] * m[dim + j];
    __shared__ double red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = red[0];
}
}  // namespace

// Entry (0, 1) of the Gram matrix of the synthesis basis (the inner-product table's row 3 at index
// 0, cuGetInnerProduct.cu:11-77): synthesise the unit coefficients 0 and 1 in FP64 and take the
// inner product of the two functions.
wp_status wp_ip_gram01_device(double* d_out, int dim, int wavelet, char bc, cudaStream_t s) {
    int levels = 0;
    while ((2 << levels) <= dim) ++levels;
    double* m = nullptr;
    WP_CUDA_TRY(cudaMallocAsync((void**)&m, sizeof(double) * 2 * (size_t)dim, s));
    unit_pair_kernel<<<wp_cdiv((size_t)2 * dim, 256), 256, 0, s>>>(m, dim);
    wp_status st = wp_dwt_axis_launch<double>(m, m, 2, dim, 1, levels, 'y', wavelet, bc, 0, s);
    if (st == WP_OK) {
        dot_pair_kernel<<<1, 256, 0, s>>>(m, d_out, dim);
        if (cudaError_t e = cudaGetLastError(); e != cudaSuccess) {
            wp_set_cuda_error(e, "gram01", __FILE__, __LINE__);
            st = WP_ERR_CUDA;
        }
    }
    cudaFreeAsync(m, s);
    return st;
}

extern "C" CUWHHD_API wp_status wp_ip_diag(double* out, int dim, int wavelet, char bc) {
    if (!out || dim < 4) { wp_set_error_msg("wp_ip_diag: bad arguments"); return WP_ERR_INVALID_ARG; }
    double* d = nullptr;
    WP_CUDA_TRY(cudaMalloc((void**)&d, sizeof(double) * dim));
    wp_status st = wp_ip_diag_device(d, dim, wavelet, bc, 0);
    if (st == WP_OK) {
        cudaError_t e = cudaMemcpy(out, d, sizeof(double) * dim, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { wp_set_cuda_error(e, "wp_ip_diag copy", __FILE__, __LINE__); st = WP_ERR_CUDA; }
    }
    cudaFree(d);
    return st;
}
