/*
 * Test infrastructure only: CPU restatement of the reference qann search path
 * (see qann_oracle.h). Each function cites the reference code it restates.
 */
#include "qann_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- exact distances: reference src/distance.cpp:66-96 (l2_distance_avx2),
 * :138-151 (inner_product_avx2). Four 8-lane accumulators over 32-float steps,
 * an 8-float step into accumulator 0, ((a0+a1)+(a2+a3)) per lane, the hsum256
 * tree ((l0+l4)+(l1+l5))+((l2+l6)+(l3+l7)), then the scalar tail, each step
 * one FMA (contracted by the release build). ------------------------------ */
static float avx2_order(const float* a, const float* b, size_t n, int l2) {
    float acc[4][8];
    memset(acc, 0, sizeof(acc));
    size_t i = 0;
    for (; i + 32 <= n; i += 32)
        for (int j = 0; j < 4; ++j)
            for (int L = 0; L < 8; ++L) {
                const size_t e = i + 8 * j + L;
                if (l2) {
                    const float d = a[e] - b[e];
                    acc[j][L] = fmaf(d, d, acc[j][L]);
                } else {
                    acc[j][L] = fmaf(a[e], b[e], acc[j][L]);
                }
            }
    for (; i + 8 <= n; i += 8)
        for (int L = 0; L < 8; ++L) {
            if (l2) {
                const float d = a[i + L] - b[i + L];
                acc[0][L] = fmaf(d, d, acc[0][L]);
            } else {
                acc[0][L] = fmaf(a[i + L], b[i + L], acc[0][L]);
            }
        }
    float s[8];
    for (int L = 0; L < 8; ++L) s[L] = (acc[0][L] + acc[1][L]) + (acc[2][L] + acc[3][L]);
    float r = ((s[0] + s[4]) + (s[1] + s[5])) + ((s[2] + s[6]) + (s[3] + s[7]));
    /* the release build vectorises the scalar tail: with 4 or more elements
     * left, four products are rounded (vmulps) and added in order; the rest
     * are fused multiply-adds */
    if (n - i >= 4) {
        for (size_t e = i; e < i + 4; ++e) {
            const float p = l2 ? (a[e] - b[e]) * (a[e] - b[e]) : a[e] * b[e];
            r = r + p;
        }
        i += 4;
    }
    for (; i < n; ++i) {
        if (l2) {
            const float d = a[i] - b[i];
            r = fmaf(d, d, r);
        } else {
            r = fmaf(a[i], b[i], r);
        }
    }
    return r;
}

float or_l2(const float* a, const float* b, size_t n) { return avx2_order(a, b, n, 1); }
float or_ip(const float* a, const float* b, size_t n) { return avx2_order(a, b, n, 0); }

/* ---- PQ tables: reference src/pq.cpp:165-223; yt is m * sd * 16 ------------- */
void or_inner_table(const float* q, const float* yt, size_t m, size_t sd, float* out) {
    for (size_t s = 0; s < m; ++s)
        for (int k = 0; k < 16; ++k) {
            float o = 0.0f;
            for (size_t j = 0; j < sd; ++j) o = fmaf(-2.0f * q[s * sd + j], yt[(s * sd + j) * 16 + k], o);
            out[s * 16 + k] = o;
        }
}

void or_list_term(const float* c, const float* yt, size_t m, size_t sd, float* out) {
    for (size_t s = 0; s < m; ++s)
        for (int k = 0; k < 16; ++k) {
            float o = 0.0f;
            for (size_t j = 0; j < sd; ++j) {
                const float y = yt[(s * sd + j) * 16 + k];
                o = fmaf(y, y + 2.0f * c[s * sd + j], o);
            }
            out[s * 16 + k] = o;
        }
}

void or_adc_table(const float* r, const float* yt, size_t m, size_t sd, float* out) {
    for (size_t s = 0; s < m; ++s)
        for (int k = 0; k < 16; ++k) {
            float o = 0.0f;
            for (size_t j = 0; j < sd; ++j) {
                const float d = r[s * sd + j] - yt[(s * sd + j) * 16 + k];
                o = fmaf(d, d, o);
            }
            out[s * 16 + k] = o;
        }
}

/* ---- LUT rounding: reference src/fast_scan.cpp:22-46 (quantize_lut_scalar),
 * :243-254 (build_quantize_lut) ------------------------------------------------- */
void or_quantize_lut(const float* table, size_t m, uint8_t* lut, float* scale, float* offset) {
    float* mins = malloc(m * sizeof(float));
    float widest = 0.0f, part[4] = {0, 0, 0, 0};
    for (size_t i = 0; i < m; ++i) {
        const float* row = table + i * 16;
        float lo = row[0], hi = row[0];
        for (int j = 1; j < 16; ++j) {
            lo = row[j] < lo ? row[j] : lo;
            hi = hi < row[j] ? row[j] : hi;
        }
        mins[i] = lo;
        part[i % 4] += lo;
        const float w = hi - lo;
        widest = widest < w ? w : widest;
    }
    *offset = (part[0] + part[1]) + (part[2] + part[3]);
    *scale = widest > 0.0f ? 63.0f / widest : 1.0f;
    for (size_t i = 0; i < m; ++i)
        for (int j = 0; j < 16; ++j) lut[i * 16 + j] = (uint8_t)nearbyintf((table[i * 16 + j] - mins[i]) * *scale);
    free(mins);
}

void or_build_quantize_lut(const float* B, const float* C, float A, size_t m, float* table, uint8_t* lut,
                           float* scale, float* offset) {
    for (size_t t = 0; t < m * 16; ++t) table[t] = B[t] + C[t];
    for (int j = 0; j < 16; ++j) table[j] += A;
    or_quantize_lut(table, m, lut, scale, offset);
}

/* ---- block sums: reference src/fast_scan.cpp:256-262, :379-385; layout
 * src/fast_scan.hpp:6-34 ------------------------------------------------------- */
static uint8_t fs_get(const uint8_t* block, size_t pos, size_t s) {
    const uint8_t b = block[s * 16 + (pos % 16)];
    return pos < 16 ? (uint8_t)(b & 15) : (uint8_t)(b >> 4);
}

void or_fast_scan_block(const uint8_t* lut, const uint8_t* block, size_t m, uint16_t* out) {
    for (size_t v = 0; v < 32; ++v) {
        uint16_t sum = 0;
        for (size_t s = 0; s < m; ++s) sum = (uint16_t)(sum + lut[s * 16 + fs_get(block, v, s)]);
        out[v] = sum;
    }
}

uint32_t or_fast_scan_block_mask(const uint8_t* lut, const uint8_t* block, size_t m, uint16_t limit, uint16_t* out) {
    or_fast_scan_block(lut, block, m, out);
    uint32_t mask = 0;
    for (size_t v = 0; v < 32; ++v)
        if (out[v] < limit) mask |= 1u << v;
    return mask;
}

/* ---- 16-centroid encoder: reference src/pq.cpp:88-116 (AVX2+FMA path) ------ */
void or_encode16(const float* r, const float* yt, size_t m, size_t sd, uint8_t* codes) {
    for (size_t s = 0; s < m; ++s) {
        float acc[16];
        for (int k = 0; k < 16; ++k) {
            const float d = r[s * sd] - yt[(s * sd) * 16 + k];
            acc[k] = d * d;
        }
        for (size_t j = 1; j < sd; ++j)
            for (int k = 0; k < 16; ++k) {
                const float d = r[s * sd + j] - yt[(s * sd + j) * 16 + k];
                acc[k] = fmaf(d, d, acc[k]);
            }
        float mn = acc[0];
        for (int k = 1; k < 16; ++k) mn = acc[k] < mn ? acc[k] : mn;
        int best = 0;
        while (acc[best] != mn) ++best;
        codes[s] = (uint8_t)best;
    }
}

/* ---- cosine rows: reference src/index.cpp:193-218 (the double sum contracted) */
int or_normalize_row(const float* x, size_t d, float* out) {
    double s = 0.0;
    for (size_t j = 0; j < d; ++j) s = fma((double)x[j], (double)x[j], s);
    const double len = sqrt(s);
    if (len == 0) return 1;
    const float scale = (float)(1.0 / len);
    for (size_t j = 0; j < d; ++j) out[j] = x[j] * scale;
    return 0;
}

/* ---- TopK: reference src/topk.hpp:26-138 --------------------------------- */
static uint32_t fkey(float f) {
    uint32_t b;
    memcpy(&b, &f, 4);
    return b ^ ((uint32_t)((int32_t)b >> 31) | 0x80000000u);
}

static float kfloat(uint32_t k) {
    const uint32_t b = (k & 0x80000000u) ? (k ^ 0x80000000u) : ~k;
    float f;
    memcpy(&f, &b, 4);
    return f;
}

typedef struct {
    size_t k, n;
    float worst;
    float* dist;
    uint32_t* slot;
    uint64_t* push;
    uint32_t* keys;
} TopK;

static void tk_init(TopK* t, size_t k) {
    t->k = k;
    t->n = 0;
    t->worst = INFINITY;
    t->dist = malloc(2 * k * sizeof(float));
    t->slot = malloc(2 * k * sizeof(uint32_t));
    t->push = malloc(2 * k * sizeof(uint64_t));
    t->keys = malloc(2 * k * sizeof(uint32_t));
}

static void tk_free(TopK* t) {
    free(t->dist);
    free(t->slot);
    free(t->push);
    free(t->keys);
}

static size_t tk_count_le(const TopK* t, uint32_t v) {
    size_t c = 0;
    for (size_t i = 0; i < t->n; ++i) c += t->keys[i] <= v;
    return c;
}

/* keeps the k smallest keys, ties at the k-th in push order */
static void tk_trim(TopK* t) {
    const size_t n = t->n;
    uint32_t lo = UINT32_MAX, hi = 0;
    for (size_t i = 0; i < n; ++i) {
        t->keys[i] = fkey(t->dist[i]);
        lo = t->keys[i] < lo ? t->keys[i] : lo;
        hi = t->keys[i] > hi ? t->keys[i] : hi;
    }
    const uint32_t x = lo ^ hi;
    int bits = 0;
    while (bits < 32 && (x >> bits) != 0) ++bits;
    uint32_t thr = bits == 32 ? 0 : lo & ~((1u << bits) - 1);
    for (int b = bits - 1; b >= 0; --b) {
        const uint32_t below = (1u << b) - 1;
        if (tk_count_le(t, thr | below) < t->k) thr |= 1u << b;
    }
    size_t ties = t->k - (thr == 0 ? 0 : tk_count_le(t, thr - 1));
    size_t w = 0;
    for (size_t i = 0; i < n; ++i) {
        const int tie = t->keys[i] == thr && ties > 0;
        t->dist[w] = t->dist[i];
        t->slot[w] = t->slot[i];
        t->push[w] = t->push[i];
        w += t->keys[i] < thr || tie;
        ties -= tie;
    }
    t->n = t->k;
    t->worst = kfloat(thr);
}

static void tk_push(TopK* t, float d, uint32_t slot, uint64_t push) {
    t->dist[t->n] = d;
    t->slot[t->n] = slot;
    t->push[t->n] = push;
    if (++t->n >= 2 * t->k) tk_trim(t);
}

typedef struct {
    uint32_t key;
    uint64_t push;
    uint32_t slot;
    float dist;
} Cand;

static int cand_cmp(const void* a, const void* b) {
    const Cand* x = a;
    const Cand* y = b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    if (x->push != y->push) return x->push < y->push ? -1 : 1;
    return 0;
}

/* ---- one IVF fast-scan query: reference src/ivf_index.cpp:421-641 -------- */
size_t or_ivf_fs_query(const float* q, size_t dim, size_t m, int mode, const float* yt, size_t sd, const float* B,
                       const float* centers, const uint8_t* codes, const uint32_t* slots, const uint64_t* offsets,
                       const uint32_t* sizes, const uint32_t* probes, const float* pterm, size_t nprobe, size_t k,
                       const uint64_t* deleted, int semantics, float* out_dist, uint32_t* out_slot) {
    const size_t T = m * 16;
    float* table = malloc(T * sizeof(float));
    float* C = malloc(T * sizeof(float));
    float* resid = malloc(dim * sizeof(float));
    uint8_t* lut = malloc(T);
    float ip_scale = 1.0f, ip_offset = 0.0f;
    if (mode == 0) or_inner_table(q, yt, m, sd, C);
    if (mode == 2 || mode == 3) {
        or_inner_table(q, yt, m, sd, table);
        if (mode == 2)
            for (size_t t = 0; t < T; ++t) table[t] *= 0.5f;
        or_quantize_lut(table, m, lut, &ip_scale, &ip_offset);
    }
    TopK top;
    tk_init(&top, k);
    size_t cap = 1024, nc = 0;
    Cand* all = semantics == 1 ? malloc(cap * sizeof(Cand)) : NULL;
    uint64_t push_base = 0;
    for (size_t p = 0; p < nprobe; ++p) {
        const uint32_t l = probes[p];
        float scale, offset;
        if (mode == 0) {
            or_build_quantize_lut(B + (size_t)l * T, C, pterm[p], m, table, lut, &scale, &offset);
        } else if (mode == 1) {
            for (size_t d = 0; d < dim; ++d) resid[d] = q[d] - centers[(size_t)l * dim + d];
            or_adc_table(resid, yt, m, sd, table);
            or_quantize_lut(table, m, lut, &scale, &offset);
        } else {
            scale = ip_scale;
            offset = ip_offset + pterm[p];
        }
        const uint32_t n = sizes[l];
        const uint8_t* lc = codes + offsets[l] * m;
        const uint32_t* ls = slots + offsets[l];
        for (uint32_t start = 0; start < n; start += 32) {
            const uint32_t cnt = n - start < 32 ? n - start : 32;
            uint32_t limit16 = 65535;
            if (semantics == 0) {
                const float lim = (top.worst - offset) * scale;
                limit16 = lim >= 65535.0f ? 65535 : lim <= 0.0f ? 0 : (uint32_t)ceilf(lim);
            }
            for (uint32_t v = 0; v < cnt; ++v) {
                const uint8_t* c = lc + (size_t)(start + v) * m;
                uint32_t sum = 0;
                for (size_t s = 0; s < m; ++s) sum += lut[s * 16 + c[s]];
                if (semantics == 0 && !(sum < limit16)) continue;
                const float dist = (float)sum / scale + offset;
                const uint32_t slot = ls[start + v];
                const int del = deleted && ((deleted[slot >> 6] >> (slot & 63)) & 1);
                if (semantics == 0) {
                    if (dist < top.worst && !del) tk_push(&top, dist, slot, push_base + start + v);
                } else if (!del) {
                    if (nc == cap) {
                        cap *= 2;
                        all = realloc(all, cap * sizeof(Cand));
                    }
                    all[nc].key = fkey(dist);
                    all[nc].push = push_base + start + v;
                    all[nc].slot = slot;
                    all[nc].dist = dist;
                    ++nc;
                }
            }
        }
        push_base += n;
    }
    size_t outn;
    if (semantics == 0) {
        if (top.n > k) tk_trim(&top);
        outn = top.n;
        Cand* kept = malloc((outn ? outn : 1) * sizeof(Cand));
        for (size_t i = 0; i < outn; ++i) {
            kept[i].key = fkey(top.dist[i]);
            kept[i].push = top.push[i];
            kept[i].slot = top.slot[i];
            kept[i].dist = top.dist[i];
        }
        qsort(kept, outn, sizeof(Cand), cand_cmp);
        for (size_t i = 0; i < outn; ++i) {
            out_dist[i] = kept[i].dist;
            out_slot[i] = kept[i].slot;
        }
        free(kept);
    } else {
        qsort(all, nc, sizeof(Cand), cand_cmp);
        outn = nc < k ? nc : k;
        for (size_t i = 0; i < outn; ++i) {
            out_dist[i] = all[i].dist;
            out_slot[i] = all[i].slot;
        }
        free(all);
    }
    tk_free(&top);
    free(table);
    free(C);
    free(resid);
    free(lut);
    return outn;
}
