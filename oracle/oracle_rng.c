/*
 * ORACLE (test infrastructure only) -- random number generators restated on the CPU.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load this code.
 * Nothing in the product library calls it.
 *
 * 1. WELL19937a with the Harase tempering, as used by EDIPIC-2D
 *    (src/WELL19937a_new.c:12-204, wrapped by src/pic2d_RandomNumberInterface.f90:32-37).
 *    The reference implements the recurrence as a six-state function-pointer machine whose
 *    only purpose is to avoid modulo arithmetic on the circular state index. Here the same
 *    published recurrence (Panneton, L'Ecuyer, Matsumoto, ACM TOMS 32(1), 2006; tempering by
 *    S. Harase) is written directly on a circular buffer: every call decrements the index
 *    i (mod 624), writes new V[i+1] and V[i] words and returns
 *    (V[i] ^ (V[i+M2+1] & 0x41180000)) * (1+2^-32) * 2^-32.
 *    The compiled reference file is the known-answer source for this restatement (the
 *    oracle/Makefile builds it in place into oracle/_ref/).
 *
 * 2. The seeding of pic2d_RandomNumberInterface.f90:39-57 (well_random_seed): a Knuth-style
 *    linear recurrence over 624 words whose shift is ISHFT(x,30), i.e. a LEFT shift on a
 *    32-bit integer, followed by set_state(state, 0, 1).
 *
 * 3. Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11 "Parallel random numbers: as easy as
 *    1, 2, 3"), the counter-based generator the GPU kernels use. Restated from the paper's
 *    round function: multipliers 0xD2511F53 / 0xCD9E8D57, Weyl key increments
 *    0x9E3779B9 / 0xBB67AE85, ten rounds.
 */
#include <stdint.h>
#include <string.h>

#define WELL_R 624
#define WELL_M1 70
#define WELL_M2 179
#define WELL_M3 449

typedef struct {
    uint32_t v[WELL_R];
    int i;
} oracle_well_t;

static uint32_t mat0pos(int t, uint32_t x) { return x ^ (x >> t); }
static uint32_t mat0neg(int t, uint32_t x) { return x ^ (x << t); }

static uint32_t at(const oracle_well_t* s, int k) { return s->v[((k % WELL_R) + WELL_R) % WELL_R]; }
static void put(oracle_well_t* s, int k, uint32_t x) { s->v[((k % WELL_R) + WELL_R) % WELL_R] = x; }

void oracle_well_set_state(oracle_well_t* s, const uint32_t* words, int index)
{
    memcpy(s->v, words, sizeof(s->v));
    s->i = index;
}

/* pic2d_RandomNumberInterface.f90:39-57 */
void oracle_well_seed(oracle_well_t* s, int32_t seed)
{
    uint32_t w[WELL_R];
    w[0] = (uint32_t)seed;
    for (int j = 1; j < WELL_R; ++j) {
        uint32_t x = w[j - 1];
        uint32_t z = x ^ (x << 30);           /* ieor(x, ishft(x,30)) on INTEGER(4) */
        w[j] = 1812433253u * z + (uint32_t)j; /* low 32 bits of the INTEGER(8) product + (j-1) for 1-based j */
    }
    oracle_well_set_state(s, w, 0);
}

/* One draw in [0,1): the WELL19937a recurrence of WELL19937a_new.c:139-203 on a circular index. */
double oracle_well_next(oracle_well_t* s)
{
    const uint32_t MASKU = 0xffffffffu >> 1; /* W - DISCARD = 1 */
    const uint32_t MASKL = ~MASKU;
    int i = s->i;
    uint32_t z0 = (at(s, i - 1) & MASKL) | (at(s, i - 2) & MASKU);
    uint32_t z1 = mat0neg(25, at(s, i)) ^ mat0pos(27, at(s, i + WELL_M1));
    uint32_t z2 = (at(s, i + WELL_M2) >> 9) ^ mat0pos(1, at(s, i + WELL_M3));
    uint32_t n1 = z1 ^ z2;
    put(s, i, n1);
    uint32_t n0 = z0 ^ mat0neg(9, z1) ^ mat0neg(21, z2) ^ mat0pos(21, n1);
    put(s, i - 1, n0);
    i = ((i - 1) % WELL_R + WELL_R) % WELL_R;
    s->i = i;
    uint32_t y = at(s, i) ^ (at(s, i + WELL_M2 + 1) & 0x41180000u);
    return (double)y * 0x1.00000001p-32;
}

/* ---------------------------------------------------------------- Philox4x32-10 */

static void mulhilo(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo)
{
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    *lo = (uint32_t)p;
}

void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4])
{
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo(0xD2511F53u, c0, &hi0, &lo0);
        mulhilo(0xCD9E8D57u, c2, &hi1, &lo1);
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n1 = lo1;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        uint32_t n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* SplitMix64 (Steele, Lea and Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014): the state
 * after n steps is s0 + n * 0x9E3779B97F4A7C15 (mod 2^64) and each output is the mix64 finaliser of the state. The
 * device cycle evaluates it at one position per particle and step for the collision decision draws. */
uint64_t oracle_mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* output n (n = 1, 2, ...) of the sequential generator seeded with s0: mix64(s0 + n gamma) */
uint64_t oracle_splitmix64_at(uint64_t s0, uint64_t n)
{
    return oracle_mix64(s0 + n * 0x9E3779B97F4A7C15ull);
}

/* the first `count` outputs of the sequential generator seeded with s0, stepped one state at a time */
void oracle_splitmix64_stream(uint64_t s0, int64_t count, uint64_t* out)
{
    uint64_t s = s0;
    for (int64_t k = 0; k < count; ++k) {
        s += 0x9E3779B97F4A7C15ull;
        out[k] = oracle_mix64(s);
    }
}
