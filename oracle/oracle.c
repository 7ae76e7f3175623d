/*
 * ORACLE -- test infrastructure only.
 *
 * A plain-C, single-purpose restatement of zeknox's polynomial-commitment
 * path, used as the checker for the CUDA library: tests, smoke() and the
 * bench's cpu_baseline leg call it; nothing in the product links it.
 *
 * Parity is pinned (tests/test_oracle.py) against
 *   - the known-answer vectors of zeknox's own tests (native/tests/tests.cu
 *     Poseidon :279-292, Poseidon2 :409-428, Keccak :164-173, Monolith
 *     :201-203, Poseidon-BN128 :492-501; Go Merkle caps
 *     wrappers/go/lib/lib_test.go:194-213), committed in tests/golden/, and
 *   - outputs of zeknox's own C++ CPU Merkle path compiled from its sources
 *     (oracle/build_ref.sh -> oracle/_ref/), committed as fixtures.
 *
 * Every routine cites the zeknox file:line whose behaviour it restates.
 * Field elements are u64, canonical in [0, p), p = 2^64 - 2^32 + 1.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ZK_CONST_TABLE static const
#include "../zeknox_b200/csrc/zk_constants.h"

typedef uint64_t u64;
typedef unsigned __int128 u128;

static const u64 P = 0xffffffff00000001ull;

/* ------------------------------------------------------------------ field */
/* ff/goldilocks.hpp:139-177 (cpp_gl64_t modulo_add / modulo_sub / reduce128),
 * restated as plain modular arithmetic with canonical results. */
/* x mod p for any 128-bit x, using 2^64 = 2^32 - 1 and 2^96 = -1 (mod p):
 * x = lo + 2^64 (h0 + 2^32 h1) = lo + h0 (2^32 - 1) - h1; the sum below is
 * < 3 * 2^64 and positive, so a few subtractions finish the reduction. */
static u64 red128(u128 x) {
    u64 lo = (u64)x, hi = (u64)(x >> 64);
    u128 r = (u128)lo + (u128)(hi & 0xffffffffull) * 0xffffffffull + P - (hi >> 32);
    while (r >= P) r -= P;
    return (u64)r;
}
u64 orc_add(u64 a, u64 b) { return red128((u128)a + b); }
u64 orc_sub(u64 a, u64 b) { return red128((u128)a + P - (b % P)); }
u64 orc_mul(u64 a, u64 b) { return red128((u128)a * b); }
u64 orc_pow(u64 a, u64 e) {
    u64 r = 1;
    a = red128(a);
    while (e) {
        if (e & 1) r = orc_mul(r, a);
        a = orc_mul(a, a);
        e >>= 1;
    }
    return r;
}
u64 orc_inv(u64 a) { return orc_pow(a, P - 2); }

/* ff/gl64_params.hpp:12-87: GROUP_GENERATOR = 7; OMEGA[k] is a primitive
 * 2^k-th root of unity, OMEGA[k] = 7^((p-1)/2^k) (scripts/gen_field_params.py
 * squares the 2^32-nd root down); OMEGA_INV[k] its inverse; DOMAIN_SIZE_INV[k]
 * = 2^-k. */
u64 orc_omega(unsigned lg) { return orc_pow(7, (P - 1) >> lg); }
u64 orc_omega_inv(unsigned lg) { return orc_inv(orc_omega(lg)); }
u64 orc_domain_size_inv(unsigned lg) { return orc_inv(orc_pow(2, lg)); }

/* --------------------------------------------------------------- Poseidon */
/* poseidon/poseidon.cu:602-791 (the naive permutation the GPU path runs):
 * 4 full rounds, 22 partial rounds, 4 full rounds; each round adds 12 round
 * constants, applies x^7 (all lanes / lane 0), then the MDS layer
 * out[r] = sum_i circ[i] * x[(i + r) % 12] + diag[r] * x[r]. */
static u64 sbox7(u64 x) {
    u64 x2 = orc_mul(x, x), x4 = orc_mul(x2, x2), x3 = orc_mul(x, x2);
    return orc_mul(x3, x4);
}
static void poseidon_mds(u64 st[12]) {
    u64 out[12];
    for (int r = 0; r < 12; r++) {
        u128 acc = 0;
        for (int i = 0; i < 12; i++) acc += (u128)st[(i + r) % 12] * ZK_POSEIDON_MDS_CIRC[i];
        acc += (u128)st[r] * ZK_POSEIDON_MDS_DIAG[r];
        out[r] = red128(acc);
    }
    memcpy(st, out, sizeof(out));
}
void orc_poseidon_permute(u64 st[12]) {
    int rnd = 0;
    for (int k = 0; k < 4; k++, rnd++) {
        for (int i = 0; i < 12; i++) st[i] = sbox7(orc_add(st[i], ZK_POSEIDON_RC[12 * rnd + i]));
        poseidon_mds(st);
    }
    for (int k = 0; k < 22; k++, rnd++) {
        for (int i = 0; i < 12; i++) st[i] = orc_add(st[i], ZK_POSEIDON_RC[12 * rnd + i]);
        st[0] = sbox7(st[0]);
        poseidon_mds(st);
    }
    for (int k = 0; k < 4; k++, rnd++) {
        for (int i = 0; i < 12; i++) st[i] = sbox7(orc_add(st[i], ZK_POSEIDON_RC[12 * rnd + i]));
        poseidon_mds(st);
    }
}

/* -------------------------------------------------------------- Poseidon2 */
/* poseidon2/poseidon2.cu:61-209: initial external layer, 4 external rounds
 * (RC, x^7 on all lanes, external layer), 22 internal rounds (RC on lane 0,
 * x^7 on lane 0, x_i <- x_i * D_i + sum), 4 external rounds.  The external
 * layer applies the 4x4 block [[5,7,1,3],[4,6,1,1],[1,3,5,7],[1,1,4,6]]
 * (apply_m_4, poseidon2.cu:64-78) to each quarter and adds the column sums. */
static void p2_m4(u64 *x) {
    static const int M[4][4] = {{5, 7, 1, 3}, {4, 6, 1, 1}, {1, 3, 5, 7}, {1, 1, 4, 6}};
    u64 o[4];
    for (int r = 0; r < 4; r++) {
        u128 acc = 0;
        for (int c = 0; c < 4; c++) acc += (u128)x[c] * M[r][c];
        o[r] = red128(acc);
    }
    memcpy(x, o, sizeof(o));
}
static void p2_external(u64 st[12]) {
    for (int i = 0; i < 12; i += 4) p2_m4(st + i);
    u64 s[4];
    for (int j = 0; j < 4; j++) s[j] = orc_add(orc_add(st[j], st[j + 4]), st[j + 8]);
    for (int i = 0; i < 12; i++) st[i] = orc_add(st[i], s[i % 4]);
}
void orc_poseidon2_permute(u64 st[12]) {
    p2_external(st);
    for (int r = 0; r < 4; r++) {
        for (int i = 0; i < 12; i++) st[i] = sbox7(orc_add(st[i], ZK_POSEIDON2_RC[12 * r + i]));
        p2_external(st);
    }
    for (int r = 4; r < 26; r++) {
        st[0] = sbox7(orc_add(st[0], ZK_POSEIDON2_RC[12 * r]));
        u64 sum = 0;
        for (int i = 0; i < 12; i++) sum = orc_add(sum, st[i]);
        for (int i = 0; i < 12; i++) st[i] = orc_add(orc_mul(st[i], ZK_POSEIDON2_DIAG[i]), sum);
    }
    for (int r = 26; r < 30; r++) {
        for (int i = 0; i < 12; i++) st[i] = sbox7(orc_add(st[i], ZK_POSEIDON2_RC[12 * r + i]));
        p2_external(st);
    }
}

/* ----------------------------------------------------------------- Keccak */
/* keccak/keccak.cu:42-112: Keccak-f[1600], 24 rounds; sponge with rate
 * 200 - 2*32 = 136 bytes, pad byte 0x01 after the message and 0x80 into the
 * last rate byte; output the first 32 bytes of the state (little-endian). */
static u64 rotl(u64 x, int s) { return s ? (x << s) | (x >> (64 - s)) : x; }
static void keccak_f(u64 a[25]) {
    for (int rnd = 0; rnd < 24; rnd++) {
        u64 c[5], d[5], b[25];
        for (int x = 0; x < 5; x++) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
        for (int x = 0; x < 5; x++) d[x] = c[(x + 4) % 5] ^ rotl(c[(x + 1) % 5], 1);
        for (int i = 0; i < 25; i++) a[i] ^= d[i % 5];
        /* rho + pi: B[y, 2x+3y] = rot(A[x, y], r[x, y]) */
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++) b[y + 5 * ((2 * x + 3 * y) % 5)] = rotl(a[x + 5 * y], ZK_KECCAK_RHO[x + 5 * y]);
        for (int y = 0; y < 5; y++)
            for (int x = 0; x < 5; x++)
                a[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
        a[0] ^= ZK_KECCAK_RC[rnd];
    }
}
void orc_keccak256(const uint8_t *in, size_t len, uint8_t out[32]) {
    u64 st[25] = {0};
    const size_t rate = 136;
    uint8_t blk[136];
    while (len >= rate) {
        for (int i = 0; i < 17; i++) {
            u64 w;
            memcpy(&w, in + 8 * i, 8);
            st[i] ^= w;
        }
        keccak_f(st);
        in += rate;
        len -= rate;
    }
    memset(blk, 0, rate);
    memcpy(blk, in, len);
    blk[len] = 0x01;
    blk[rate - 1] |= 0x80;
    for (int i = 0; i < 17; i++) {
        u64 w;
        memcpy(&w, blk + 8 * i, 8);
        st[i] ^= w;
    }
    keccak_f(st);
    memcpy(out, st, 32);
}

/* --------------------------------------------------------------- Monolith */
/* monolith/monolith.cu:117-233 (Monolith-64, width 12, 6 rounds):
 * state = (lo, hi) with hi in {0, 1} (a 65-bit lane); concrete(rc) sets lane r
 * to (sum_c M[r][c] (lo_c + 2^64 hi_c) + rc[r]) mod p, canonical, hi = 0, with
 * M circulant (row r column c = ROW[(c - r) mod 12]); bars apply the byte-wise
 * Bar S-box to lanes 0..3 (per byte: y = rotl1(x ^ (rotl1(~x) & rotl2(x) &
 * rotl3(x)))); bricks (Feistel type 3) add, from lane 11 down to lane 1, the
 * square mod p of the lane below (its value before the layer) as a 64-bit sum
 * whose carry goes to hi.  Permutation: concrete(rc0); then for r = 1..6
 * bars, bricks, concrete(rc_r). */
static u64 mono_rotl_bytes(u64 x, int k) {
    u64 out = 0;
    for (int b = 0; b < 8; b++) {
        unsigned v = (unsigned)(x >> (8 * b)) & 0xff;
        v = ((v << k) | (v >> (8 - k))) & 0xff;
        out |= (u64)v << (8 * b);
    }
    return out;
}
static u64 mono_bar(u64 x) {
    u64 t = x ^ (mono_rotl_bytes(~x, 1) & mono_rotl_bytes(x, 2) & mono_rotl_bytes(x, 3));
    return mono_rotl_bytes(t, 1);
}
static void mono_concrete(u64 lo[12], unsigned hi[12], const u64 *rc) {
    u64 out[12];
    for (int r = 0; r < 12; r++) {
        u128 acc = rc[r];
        for (int c = 0; c < 12; c++) {
            u128 m = ZK_MONOLITH_MDS_ROW[(c - r + 12) % 12];
            acc += m * lo[c] + ((m * hi[c]) << 64);
        }
        out[r] = red128(acc);
    }
    for (int r = 0; r < 12; r++) {
        lo[r] = out[r];
        hi[r] = 0;
    }
}
void orc_monolith_permute(u64 st[12]) {
    unsigned hi[12] = {0};
    mono_concrete(st, hi, ZK_MONOLITH_RC);
    for (int r = 1; r <= 6; r++) {
        for (int i = 0; i < 4; i++) st[i] = mono_bar(st[i]);
        for (int i = 11; i > 0; i--) {
            u64 sq = orc_mul(st[i - 1], st[i - 1]);
            u64 s = st[i] + sq;
            hi[i] = s < sq;
            st[i] = s;
        }
        mono_concrete(st, hi, ZK_MONOLITH_RC + 12 * r);
    }
}

/* --------------------------------------------------------- Poseidon-BN128 */
/* poseidon/poseidon_bn128.cu:111-193 with the field of element_bn128.cu:
 * circomlib's Poseidon over the BN254 scalar field r, t = 5, 8 full and 60
 * partial rounds in the optimised form (constants C, M, P, S in Montgomery
 * form, R = 2^256).  The 12 Goldilocks lanes (canonical) become 4 field
 * elements x_i = in[3i+2] + in[3i+1] 2^64 + in[3i] 2^128; the state is
 * (0, x_0..x_3); after the permutation lane i of the output is limb 2 - (i mod 3)
 * of state element i / 3, reduced mod p once. */
static const u64 BN_R[4] = {0x43e1f593f0000001ull, 0x2833e84879b97091ull, 0xb85045b68181585dull,
                            0x30644e72e131a029ull};
static const u64 BN_NINV = 0xc2e1f593efffffffull;  /* -r^-1 mod 2^64 */
static const u64 BN_R2[4] = {0x1bb8e645ae216da7ull, 0x53fe3ab1e35c59e3ull, 0x8c49833d53bb8085ull,
                             0x0216d0b17f4e44a5ull};  /* 2^512 mod r */
static int bn_geq(const u64 a[4], const u64 b[4]) {
    for (int i = 3; i >= 0; i--)
        if (a[i] != b[i]) return a[i] > b[i];
    return 1;
}
static void bn_sub_r(u64 a[4]) {
    u64 borrow = 0;
    for (int i = 0; i < 4; i++) {
        u128 d = (u128)a[i] - BN_R[i] - borrow;
        a[i] = (u64)d;
        borrow = (u64)(d >> 64) ? 1 : 0;
    }
}
static void bn_add(u64 z[4], const u64 x[4], const u64 y[4]) {
    u64 c = 0, t[4];
    for (int i = 0; i < 4; i++) {
        u128 s = (u128)x[i] + y[i] + c;
        t[i] = (u64)s;
        c = (u64)(s >> 64);
    }
    if (bn_geq(t, BN_R)) bn_sub_r(t);  /* x, y < r < 2^254: no carry out */
    memcpy(z, t, 32);
}
/* Montgomery product x y / 2^256 mod r (CIOS), fully reduced. */
static void bn_mul(u64 z[4], const u64 x[4], const u64 y[4]) {
    u64 t[6] = {0};
    for (int i = 0; i < 4; i++) {
        u64 c = 0;
        for (int j = 0; j < 4; j++) {
            u128 v = (u128)x[j] * y[i] + t[j] + c;
            t[j] = (u64)v;
            c = (u64)(v >> 64);
        }
        u128 v = (u128)t[4] + c;
        t[4] = (u64)v;
        t[5] = (u64)(v >> 64);
        u64 m = t[0] * BN_NINV;
        v = (u128)m * BN_R[0] + t[0];
        c = (u64)(v >> 64);
        for (int j = 1; j < 4; j++) {
            v = (u128)m * BN_R[j] + t[j] + c;
            t[j - 1] = (u64)v;
            c = (u64)(v >> 64);
        }
        v = (u128)t[4] + c;
        t[3] = (u64)v;
        t[4] = t[5] + (u64)(v >> 64);
    }
    u64 out[4] = {t[0], t[1], t[2], t[3]};
    if (t[4] || bn_geq(out, BN_R)) bn_sub_r(out);
    memcpy(z, out, 32);
}
static void bn_exp5(u64 x[4]) {
    u64 x2[4], x4[4];
    bn_mul(x2, x, x);
    bn_mul(x4, x2, x2);
    bn_mul(x, x4, x);
}
/* new[i] = sum_j m[j][i] state[j] */
static void bn_mix(u64 st[5][4], const u64 *m) {
    u64 out[5][4];
    for (int i = 0; i < 5; i++) {
        u64 acc[4] = {0}, prod[4];
        for (int j = 0; j < 5; j++) {
            bn_mul(prod, m + 4 * (5 * j + i), st[j]);
            bn_add(acc, acc, prod);
        }
        memcpy(out[i], acc, 32);
    }
    memcpy(st, out, sizeof(out));
}
static void bn_ark(u64 st[5][4], int it) {
    for (int i = 0; i < 5; i++) bn_add(st[i], st[i], ZK_BN128_C + 4 * (it + i));
}
void orc_poseidon_bn128_permute(u64 lanes[12]) {
    u64 st[5][4];
    memset(st, 0, sizeof(st));
    for (int i = 0; i < 4; i++) {
        u64 x[4] = {lanes[3 * i + 2] % P, lanes[3 * i + 1] % P, lanes[3 * i] % P, 0};
        bn_mul(st[i + 1], x, BN_R2);  /* to Montgomery form */
    }
    bn_ark(st, 0);
    for (int r = 0; r < 3; r++) {
        for (int i = 0; i < 5; i++) bn_exp5(st[i]);
        bn_ark(st, 5 * (r + 1));
        bn_mix(st, ZK_BN128_M);
    }
    for (int i = 0; i < 5; i++) bn_exp5(st[i]);
    bn_ark(st, 20);
    bn_mix(st, ZK_BN128_P);
    for (int r = 0; r < 60; r++) {
        bn_exp5(st[0]);
        bn_add(st[0], st[0], ZK_BN128_C + 4 * (25 + r));
        const u64 *sp = ZK_BN128_S + 4 * 9 * r;
        u64 acc[4] = {0}, prod[4];
        for (int j = 0; j < 5; j++) {
            bn_mul(prod, sp + 4 * j, st[j]);
            bn_add(acc, acc, prod);
        }
        for (int k = 1; k < 5; k++) {
            bn_mul(prod, st[0], sp + 4 * (5 + k - 1));
            bn_add(st[k], st[k], prod);
        }
        memcpy(st[0], acc, 32);
    }
    for (int r = 0; r < 3; r++) {
        for (int i = 0; i < 5; i++) bn_exp5(st[i]);
        bn_ark(st, 85 + 5 * r);
        bn_mix(st, ZK_BN128_M);
    }
    for (int i = 0; i < 5; i++) bn_exp5(st[i]);
    bn_mix(st, ZK_BN128_M);
    const u64 one[4] = {1, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
        u64 v[4];
        bn_mul(v, st[i], one);  /* out of Montgomery form */
        for (int k = 0; k < 3; k++) {
            u64 w = v[2 - k];
            lanes[3 * i + k] = w >= P ? w - P : w;
        }
    }
}

/* ---------------------------------------------------------------- hashers */
enum { H_POSEIDON = 0, H_KECCAK = 1, H_POSEIDON_BN128 = 2, H_POSEIDON2 = 3, H_MONOLITH = 4 };

/* Sponge of poseidon/poseidon_permutation.cuh:226-276 (GPU) and
 * poseidon_permutation.hpp:84-139 (CPU): width 12, rate 8, overwrite mode.
 * n <= 4: copy and zero-pad (no permutation).  Otherwise for each 8-element
 * chunk overwrite lanes 0..len-1 (a short final chunk leaves the other lanes
 * as they are) and permute; the digest is lanes 0..3. */
static void sponge_hash_one(void (*perm)(u64 *), const u64 *in, u64 n, u64 out[4]) {
    if (n <= 4) {
        u64 i = 0;
        for (; i < n; i++) out[i] = in[i];
        for (; i < 4; i++) out[i] = 0;
        return;
    }
    u64 st[12] = {0};
    for (u64 idx = 0; idx < n; idx += 8) {
        u64 len = n - idx < 8 ? n - idx : 8;
        for (u64 j = 0; j < len; j++) st[j] = in[idx + j];
        perm(st);
    }
    memcpy(out, st, 32);
}
static void sponge_hash_two(void (*perm)(u64 *), const u64 *l, const u64 *r, u64 out[4]) {
    u64 st[12] = {0};
    memcpy(st, l, 32);
    memcpy(st + 4, r, 32);
    perm(st);
    memcpy(out, st, 32);
}
/* keccak/keccak.cu:116-135: n < 4 copies n words and leaves the rest of the
 * digest untouched; otherwise keccak256 over the 8n little-endian bytes,
 * then digest[3] &= 0xff.  hash_two hashes left[0..25) || right[0..25). */
static void keccak_hash_one(const u64 *in, u64 n, u64 out[4]) {
    if (n < 4) {
        memcpy(out, in, n * 8);
        return;
    }
    orc_keccak256((const uint8_t *)in, n * 8, (uint8_t *)out);
    out[3] &= 0xff;
}
static void keccak_hash_two(const u64 *l, const u64 *r, u64 out[4]) {
    uint8_t buf[50];
    memcpy(buf, l, 25);
    memcpy(buf + 25, r, 25);
    orc_keccak256(buf, 50, (uint8_t *)out);
    out[3] &= 0xff;
}

int orc_hash_one(int ht, const u64 *in, u64 n, u64 out[4]) {
    switch (ht) {
    case H_POSEIDON: sponge_hash_one(orc_poseidon_permute, in, n, out); return 0;
    case H_POSEIDON2: sponge_hash_one(orc_poseidon2_permute, in, n, out); return 0;
    case H_MONOLITH: sponge_hash_one(orc_monolith_permute, in, n, out); return 0;
    case H_POSEIDON_BN128: sponge_hash_one(orc_poseidon_bn128_permute, in, n, out); return 0;
    case H_KECCAK: keccak_hash_one(in, n, out); return 0;
    default: return -1;
    }
}
int orc_hash_two(int ht, const u64 *l, const u64 *r, u64 out[4]) {
    switch (ht) {
    case H_POSEIDON: sponge_hash_two(orc_poseidon_permute, l, r, out); return 0;
    case H_POSEIDON2: sponge_hash_two(orc_poseidon2_permute, l, r, out); return 0;
    case H_MONOLITH: sponge_hash_two(orc_monolith_permute, l, r, out); return 0;
    case H_POSEIDON_BN128: sponge_hash_two(orc_poseidon_bn128_permute, l, r, out); return 0;
    case H_KECCAK: keccak_hash_two(l, r, out); return 0;
    default: return -1;
    }
}

/* ----------------------------------------------------------------- Merkle */
/* merkle/merkle.cu:166-244 (the GPU driver the C ABI runs):
 *  - n_caps == n_leaves: cap[i] = H1(leaf i); digests untouched.
 *  - subtree of L_s = n_leaves >> cap_height leaves, D_s = n_digests >> cap_height
 *    digests; L_s == 1: cap[i] = H1(leaf i).  L_s == 2: digest[i] = H1(leaf i),
 *    cap[s] = H2(digest[s D_s], digest[s D_s + 1]).
 *  - general: subtree s, leaf j -> digest s D_s + (D_s - L_s) + j; internal
 *    node i of subtree s (linear index inside the subtree) has children
 *    2(i+1), 2(i+1)+1; level widths 2^r at offsets 2^r - 2; cap[s] =
 *    H2(node 0, node 1). */
int orc_merkle_fill(u64 *digests, u64 *cap, const u64 *leaves, u64 n_digests, u64 n_caps,
                    u64 n_leaves, u64 leaf_size, u64 cap_height, int ht) {
    if (ht < H_POSEIDON || ht > H_MONOLITH) return -1;
    if (n_caps == n_leaves) {
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)n_leaves; i++)
            orc_hash_one(ht, leaves + i * leaf_size, leaf_size, cap + 4 * i);
        return 0;
    }
    u64 Ds = n_digests >> cap_height, Ls = n_leaves >> cap_height;
    if (Ls == 1) {
        for (u64 i = 0; i < n_leaves; i++) orc_hash_one(ht, leaves + i * leaf_size, leaf_size, cap + 4 * i);
        return 0;
    }
    if (Ls == 2) {
        for (u64 i = 0; i < n_leaves; i++) orc_hash_one(ht, leaves + i * leaf_size, leaf_size, digests + 4 * i);
        for (u64 s = 0; s < n_caps; s++) orc_hash_two(ht, digests + 4 * s * Ds, digests + 4 * (s * Ds + 1), cap + 4 * s);
        return 0;
    }
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n_leaves; i++) {
        u64 s = i / Ls, j = i % Ls;
        orc_hash_one(ht, leaves + i * leaf_size, leaf_size, digests + 4 * (s * Ds + (Ds - Ls) + j));
    }
    for (u64 w = Ls / 2; w >= 2; w /= 2) {
        u64 off = w - 2;
#pragma omp parallel for schedule(static)
        for (long long t = 0; t < (long long)(w * n_caps); t++) {
            u64 s = t / w, i = off + t % w;
            u64 *base = digests + 4 * s * Ds;
            orc_hash_two(ht, base + 4 * (2 * (i + 1)), base + 4 * (2 * (i + 1) + 1), base + 4 * i);
        }
    }
    for (u64 s = 0; s < n_caps; s++) orc_hash_two(ht, digests + 4 * s * Ds, digests + 4 * (s * Ds + 1), cap + 4 * s);
    return 0;
}

/* -------------------------------------------------------------------- NTT */
static u64 bitrev(u64 x, unsigned bits) {
    u64 r = 0;
    for (unsigned i = 0; i < bits; i++) r |= ((x >> i) & 1) << (bits - 1 - i);
    return r;
}
/* Plain transform X[k] = sum_i a[i] w^(ik), w = OMEGA[lg] (forward) or
 * OMEGA_INV[lg] (inverse), natural order in and out, no scaling.  Computed
 * by bit-reversal + iterative radix-2 Cooley-Tukey. */
void orc_ntt_raw(u64 *a, unsigned lg, int inverse) {
    u64 n = 1ull << lg;
    for (u64 i = 0; i < n; i++) {
        u64 j = bitrev(i, lg);
        if (i < j) {
            u64 t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
    for (unsigned s = 1; s <= lg; s++) {
        u64 m = 1ull << s, h = m >> 1;
        u64 wm = inverse ? orc_omega_inv(s) : orc_omega(s);
        u64 *tw = (u64 *)malloc(h * sizeof(u64));
        tw[0] = 1;
        for (u64 j = 1; j < h; j++) tw[j] = orc_mul(tw[j - 1], wm);
        for (u64 k = 0; k < n; k += m)
            for (u64 j = 0; j < h; j++) {
                u64 u = a[k + j], v = orc_mul(a[k + j + h], tw[j]);
                a[k + j] = orc_add(u, v);
                a[k + j + h] = orc_sub(u, v);
            }
        free(tw);
    }
}

/* ntt/ntt.cu:106-158 + :253-309 (batch_ntt):
 *  forward: [x_i *= coset_i if with_coset]; X = NTT_w(x), natural order.
 *  inverse: y = NTT_{w^-1}(x) natural order; [y_i *= coset_i if with_coset];
 *           y_i *= 2^-lg.
 * coset_i = coset_gen^i (the table init_coset writes, ntt.cu:228-239). */
void orc_batch_ntt(u64 *inout, unsigned lg, int inverse, unsigned batches, int with_coset, u64 coset_gen) {
    u64 n = 1ull << lg;
#pragma omp parallel for schedule(dynamic)
    for (long long b = 0; b < (long long)batches; b++) {
        u64 *a = inout + b * n;
        if (!inverse) {
            if (with_coset) {
                u64 g = 1;
                for (u64 i = 0; i < n; i++, g = orc_mul(g, coset_gen)) a[i] = orc_mul(a[i], g);
            }
            orc_ntt_raw(a, lg, 0);
        } else {
            orc_ntt_raw(a, lg, 1);
            u64 ninv = orc_domain_size_inv(lg);
            u64 g = 1;
            for (u64 i = 0; i < n; i++) {
                if (with_coset) {
                    a[i] = orc_mul(a[i], g);
                    g = orc_mul(g, coset_gen);
                }
                a[i] = orc_mul(a[i], ninv);
            }
        }
    }
}

/* ntt/ntt.cu:477-564 (batch_lde): zero-extend each of the `batches` rows from
 * 2^lg_n to N = 2^(lg_n + rate_bits) elements (kernels.cu:40-60), then the
 * size-N batch_ntt above on the extended rows. */
void orc_batch_lde(u64 *out, const u64 *in, unsigned lg_n, unsigned rate_bits, int inverse, unsigned batches,
                   int with_coset, u64 coset_gen) {
    u64 n = 1ull << lg_n, N = n << rate_bits;
    for (u64 b = 0; b < batches; b++) {
        memcpy(out + b * N, in + b * n, n * sizeof(u64));
        memset(out + b * N + n, 0, (N - n) * sizeof(u64));
    }
    orc_batch_ntt(out, lg_n + rate_bits, inverse, batches, with_coset, coset_gen);
}

/* ntt/kernels.cu:94-135 (transpose_rev_kernel): out[rev_lg(k)][b] = in[b][k]
 * for b < batches, k < 2^lg_n (equivalently out[k][b] = in[b][rev(k)]). */
void orc_transpose_rev(u64 *out, const u64 *in, unsigned lg_n, unsigned batches) {
    u64 n = 1ull << lg_n;
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < (long long)n; k++) {
        u64 r = bitrev(k, lg_n);
        for (u64 b = 0; b < batches; b++) out[r * batches + b] = in[b * n + k];
    }
}

/* -------------------------------------------------------------------- FRI */
/* One folding step of the FRI commit phase over GF(p^2) = GF(p)[X]/(X^2 - 7),
 * the quadratic extension of Goldilocks (W = 7).  The FRI prover that consumes
 * zeknox's commitments is Plonky2's (okx/plonky2, rev 9a917ba2, the git
 * dependency of wrappers/rust/Cargo.toml:43-44, not present here): each round
 * reduces the coefficient vector by `arity`, coefficient j of the result being
 * sum_t beta^t c[j*arity + t] ("reduce_with_powers").  Restated by Horner's
 * rule from the highest power down.  Split layout in and out: row 0 real
 * parts, row 1 X parts.  Parity against Plonky2 is unpinned (no copy of it). */
static void ext_mul(u64 a0, u64 a1, u64 b0, u64 b1, u64 *c0, u64 *c1) {
    u64 r0 = orc_add(orc_mul(a0, b0), orc_mul(7, orc_mul(a1, b1)));
    u64 r1 = orc_add(orc_mul(a0, b1), orc_mul(a1, b0));
    *c0 = r0;
    *c1 = r1;
}
void orc_fri_fold(u64 *out, const u64 *in, u64 n_in, unsigned arity_bits, u64 b0, u64 b1) {
    u64 a = 1ull << arity_bits, n_out = n_in >> arity_bits;
    for (u64 j = 0; j < n_out; j++) {
        u64 r0 = 0, r1 = 0;
        for (u64 t = a; t-- > 0;) {
            ext_mul(r0, r1, b0, b1, &r0, &r1);
            r0 = orc_add(r0, in[j * a + t]);
            r1 = orc_add(r1, in[n_in + j * a + t]);
        }
        out[j] = r0;
        out[n_out + j] = r1;
    }
}
