/* H.261 variable-length code tables for the device bitstream writer.
 *
 * The codes are the standard's (ITU-T H.261 Tables 1-5), the same values
 * the reference's src/h261_tables.c holds; the writer must reproduce the
 * reference's bytes, so nothing here may differ from the standard.  Layouts
 * are ours: (length << 8) | code in 16 bits, 0 = no entry. */
#pragma once

#include <cstdint>

namespace h261b {

#define VLC(code, len) (uint16_t)(((len) << 8) | (code))

/* TCOEFF without the sign bit, run 0..26 x level 0..15 (level 0 unused);
 * 0 = send with the 20-bit escape */
static __device__ __constant__ uint16_t c_vlc_tcoeff[27][16] = {
    { 0, VLC(3, 2), VLC(4, 4), VLC(5, 5), VLC(6, 7), VLC(38, 8), VLC(33, 8), VLC(10, 10), VLC(29, 12),
      VLC(24, 12), VLC(19, 12), VLC(16, 12), VLC(26, 13), VLC(25, 13), VLC(24, 13), VLC(23, 13) },
    { 0, VLC(3, 3), VLC(6, 6), VLC(37, 8), VLC(12, 10), VLC(27, 12), VLC(22, 13), VLC(21, 13) },
    { 0, VLC(5, 4), VLC(4, 7), VLC(11, 10), VLC(20, 12), VLC(20, 13) },
    { 0, VLC(7, 5), VLC(36, 8), VLC(28, 12), VLC(19, 13) },
    { 0, VLC(6, 5), VLC(15, 10), VLC(18, 12) },
    { 0, VLC(7, 6), VLC(9, 10), VLC(18, 13) },
    { 0, VLC(5, 6), VLC(30, 12) },
    { 0, VLC(4, 6), VLC(21, 12) },
    { 0, VLC(7, 7), VLC(17, 12) },
    { 0, VLC(5, 7), VLC(17, 13) },
    { 0, VLC(39, 8), VLC(16, 13) },
    { 0, VLC(35, 8) }, { 0, VLC(34, 8) }, { 0, VLC(32, 8) }, { 0, VLC(14, 10) }, { 0, VLC(13, 10) },
    { 0, VLC(8, 10) }, { 0, VLC(31, 12) }, { 0, VLC(26, 12) }, { 0, VLC(25, 12) }, { 0, VLC(23, 12) },
    { 0, VLC(22, 12) }, { 0, VLC(31, 13) }, { 0, VLC(30, 13) }, { 0, VLC(29, 13) }, { 0, VLC(28, 13) },
    { 0, VLC(27, 13) },
};

/* MBA, address increment 1..33 */
static __device__ __constant__ uint16_t c_vlc_mba[34] = {
    0,           VLC(1, 1),   VLC(3, 3),   VLC(2, 3),   VLC(3, 4),   VLC(2, 4),   VLC(3, 5),
    VLC(2, 5),   VLC(7, 7),   VLC(6, 7),   VLC(11, 8),  VLC(10, 8),  VLC(9, 8),   VLC(8, 8),
    VLC(7, 8),   VLC(6, 8),   VLC(23, 10), VLC(22, 10), VLC(21, 10), VLC(20, 10), VLC(19, 10),
    VLC(18, 10), VLC(35, 11), VLC(34, 11), VLC(33, 11), VLC(32, 11), VLC(31, 11), VLC(30, 11),
    VLC(29, 11), VLC(28, 11), VLC(27, 11), VLC(26, 11), VLC(25, 11), VLC(24, 11),
};

/* MVD by magnitude 0..16 of the wrapped difference: the negative value's
 * code (the positive value's is one less; 0 has the code 1) */
static __device__ __constant__ uint16_t c_vlc_mvd[17] = {
    VLC(1, 1),   VLC(3, 3),   VLC(3, 4),   VLC(3, 5),   VLC(7, 7),   VLC(11, 8),
    VLC(9, 8),   VLC(7, 8),   VLC(23, 10), VLC(21, 10), VLC(19, 10), VLC(35, 11),
    VLC(33, 11), VLC(31, 11), VLC(29, 11), VLC(27, 11), VLC(25, 11),
};

/* CBP 1..63 */
static __device__ __constant__ uint16_t c_vlc_cbp[64] = {
    0,          VLC(11, 5), VLC(9, 5),  VLC(13, 6), VLC(13, 4), VLC(23, 7), VLC(19, 7), VLC(31, 8),
    VLC(12, 4), VLC(22, 7), VLC(18, 7), VLC(30, 8), VLC(19, 5), VLC(27, 8), VLC(23, 8), VLC(19, 8),
    VLC(11, 4), VLC(21, 7), VLC(17, 7), VLC(29, 8), VLC(17, 5), VLC(25, 8), VLC(21, 8), VLC(17, 8),
    VLC(15, 6), VLC(15, 8), VLC(13, 8), VLC(3, 9),  VLC(15, 5), VLC(11, 8), VLC(7, 8),  VLC(7, 9),
    VLC(10, 4), VLC(20, 7), VLC(16, 7), VLC(28, 8), VLC(14, 6), VLC(14, 8), VLC(12, 8), VLC(2, 9),
    VLC(16, 5), VLC(24, 8), VLC(20, 8), VLC(16, 8), VLC(14, 5), VLC(10, 8), VLC(6, 8),  VLC(6, 9),
    VLC(18, 5), VLC(26, 8), VLC(22, 8), VLC(18, 8), VLC(13, 5), VLC(9, 8),  VLC(5, 8),  VLC(5, 9),
    VLC(12, 5), VLC(8, 8),  VLC(4, 8),  VLC(4, 9),  VLC(7, 3),  VLC(10, 5), VLC(8, 5),  VLC(12, 6),
};

#undef VLC

/* MTYPE lengths (every code is a single 1 after zeros), indexed by the
 * reference's macroblock type numbers 0..9 (src/h261_types.h:15-24) */
enum {
    MT_INTRA = 0, MT_INTRA_MQ, MT_INTER, MT_INTER_MQ, MT_MC, MT_MC_CBP, MT_MC_CBP_MQ,
    MT_MC_FIL, MT_MC_FIL_CBP, MT_MC_FIL_CBP_MQ
};
static __device__ __constant__ uint8_t c_vlc_mtype_len[10] = { 4, 7, 1, 5, 9, 8, 10, 3, 2, 6 };

/* zig-zag index of coefficient (vertical frequency v, horizontal u): the
 * diagonal d = u + v starts at d(d+1)/2 (or 64 - (15-d)(16-d)/2 past the
 * main anti-diagonal); odd diagonals run with increasing v, even ones with
 * decreasing v -- the transmission order of H.261 */
__host__ __device__ constexpr int zigzag_index(int v, int u)
{
    return (u + v < 8 ? ((u + v) * (u + v + 1)) >> 1 : 64 - (((15 - u - v) * (16 - u - v)) >> 1)) +
           (((u + v) & 1) ? v - (u + v < 8 ? 0 : u + v - 7) : (u + v < 8 ? u + v : 7) - v);
}

/* column-major index (u * 8 + v) of the k-th coefficient sent, generated
 * from zigzag_index at compile time */
struct ZigzagTable {
    uint8_t cm[64];
};
__host__ __device__ constexpr ZigzagTable make_zigzag_table()
{
    ZigzagTable t{};
    for (int v = 0; v < 8; v++)
        for (int u = 0; u < 8; u++)
            t.cm[zigzag_index(v, u)] = (uint8_t)(u * 8 + v);
    return t;
}
static __device__ __constant__ ZigzagTable c_zigzag_cm = make_zigzag_table();

/* bits of one non-DC coefficient sent after `run` zeros: table code plus
 * sign, or the escape */
__device__ __forceinline__ int tcoeff_bits(int run, int level)
{
    const int a = level < 0 ? -level : level;
    const int e = (run <= 26 && a <= 15) ? (c_vlc_tcoeff[run][a] >> 8) : 0;
    return e ? e + 1 : 20;
}

} // namespace h261b
