/*
 * Test infrastructure only: this project's CPU restatement of the reference
 * qann search path, used by tests/ and bench.py's CPU baseline as the checker.
 * Nothing in qann_b200 links or calls it.
 *
 * Arithmetic follows the reference's x86 release build (GCC, C++20, -O3
 * -mavx2 -mfma; reference CMakeLists.txt:63-68). GCC contracts `x += a * b`
 * into one fused multiply-add by default in C++ (-ffp-contract=fast), so the
 * functions below call fmaf/fma exactly where that build fuses; this file
 * itself is compiled with -ffp-contract=off so nothing else is fused.
 * Parity of this restatement is pinned against the reference library built
 * from its own sources (oracle/_ref) and the reference's golden files.
 */
#ifndef QANN_ORACLE_H
#define QANN_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

float or_l2(const float* a, const float* b, size_t n);
float or_ip(const float* a, const float* b, size_t n);
void or_inner_table(const float* q, const float* yt, size_t m, size_t sd, float* out);
void or_list_term(const float* c, const float* yt, size_t m, size_t sd, float* out);
void or_adc_table(const float* r, const float* yt, size_t m, size_t sd, float* out);
void or_quantize_lut(const float* table, size_t m, uint8_t* lut, float* scale, float* offset);
void or_build_quantize_lut(const float* B, const float* C, float A, size_t m, float* table, uint8_t* lut,
                           float* scale, float* offset);
void or_fast_scan_block(const uint8_t* lut, const uint8_t* block, size_t m, uint16_t* out);
uint32_t or_fast_scan_block_mask(const uint8_t* lut, const uint8_t* block, size_t m, uint16_t limit, uint16_t* out);
void or_encode16(const float* residual, const float* yt, size_t m, size_t sd, uint8_t* codes);
int or_normalize_row(const float* x, size_t d, float* out);

/* One IVF fast-scan query. Lists are given in plain form: list l holds
 * sizes[l] vectors starting at vector offsets[l] of `codes` (m bytes each,
 * one code per byte) and `slots`. mode: 0 L2 with precomputed tables B
 * (nlist * m * 16), 1 L2 with per-list ADC tables, 2 inner product, 3 cosine
 * scored by inner product. probes: the query's nprobe lists nearest first,
 * with `pterm` their term (A, or the cosine base). deleted: slot bitmap or
 * NULL. semantics: 0 = the reference's sequential TopK with its per-block
 * limit16 pre-filter (reference src/ivf_index.cpp:466-499), 1 = the k
 * smallest by (distance, push order) with no pre-filter. Writes up to k
 * (distance, slot) pairs sorted by key and push order; returns the count. */
size_t or_ivf_fs_query(const float* q, size_t dim, size_t m, int mode, const float* yt, size_t sd, const float* B,
                       const float* centers, const uint8_t* codes, const uint32_t* slots, const uint64_t* offsets,
                       const uint32_t* sizes, const uint32_t* probes, const float* pterm, size_t nprobe, size_t k,
                       const uint64_t* deleted, int semantics, float* out_dist, uint32_t* out_slot);

#ifdef __cplusplus
}
#endif

#endif
