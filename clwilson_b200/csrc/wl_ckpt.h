// wl_ckpt.h -- checkpoint files of the clwilson program in the reference's
// format (cl_wilson.h:22-25, cl_wilson.cpp:110-288): the workStatus header,
// then one (s0, s1) pair per test prime, the running products in the
// reference's Montgomery form (R = 2^64 mod p^2, base-p digits), and the
// additive state_sum; stateA.ckp and stateB.ckp written alternately.
// Host code only (no CUDA).
#pragma once
#include <cstdint>
#include <cstdio>
#include <vector>

static const char* const STATE_FILENAME_A = "stateA.ckp";
static const char* const STATE_FILENAME_B = "stateB.ckp";

typedef unsigned __int128 u128;

// The checkpoint header, byte for byte the reference's workStatus (cl_wilson.h:22-25).
struct WorkStatus {
    uint64_t pmin, pmax, currp, trickle, state_sum, totalcount;
    uint32_t tpcount, done;
};
static_assert(sizeof(WorkStatus) == 56, "workStatus layout");

// The reference keeps each row's running product in Montgomery form with
// R = 2^64 mod p^2, as base-p digits (kernels/common.cl:120-130); the engine
// returns plain values.  Conversion: multiply or divide by 2^64 mod p^2.
inline void to_reference(uint64_t p, uint64_t s0, uint64_t s1, uint64_t* r0, uint64_t* r1) {
    const u128 n = (u128)p * p;
    u128 x = (u128)s1 * p + s0;
    for (int i = 0; i < 64; ++i) {
        x <<= 1;
        if (x >= n) x -= n;
    }
    *r0 = (uint64_t)(x % p);
    *r1 = (uint64_t)(x / p);
}

inline void from_reference(uint64_t p, uint64_t r0, uint64_t r1, uint64_t* s0, uint64_t* s1) {
    const u128 n = (u128)p * p;
    u128 x = ((u128)r1 * p + r0) % n;
    for (int i = 0; i < 64; ++i) x = (x & 1) ? (x + n) >> 1 : x >> 1;
    *s0 = (uint64_t)(x % p);
    *s1 = (uint64_t)(x / p);
}

inline uint64_t state_checksum(const WorkStatus& st, const std::vector<uint64_t>& res) {
    uint64_t sum = st.pmin + st.pmax + st.currp + st.trickle + st.totalcount + st.tpcount + st.done;
    for (uint32_t i = 0; i < st.tpcount; ++i) sum += res[2 * i] + res[2 * i + 1];
    return sum;
}

// write_state: the header then tpcount residue pairs, alternating A and B
inline void write_state(bool& write_a_next, WorkStatus& st, const std::vector<uint64_t>& ref_res) {
    st.state_sum = state_checksum(st, ref_res);
    const char* name = write_a_next ? STATE_FILENAME_A : STATE_FILENAME_B;
    FILE* out = fopen(name, "wb");
    if (!out) {
        fprintf(stderr, "Cannot open %s !!!\n", name);
        return;
    }
    bool ok = fwrite(&st, sizeof(WorkStatus), 1, out) == 1 &&
              fwrite(ref_res.data(), 16, st.tpcount, out) == st.tpcount;
    if (!ok) fprintf(stderr, "Cannot write checkpoint to file. Continuing...\n");
    if (fclose(out) == 0 && ok) write_a_next = !write_a_next;
}

// read_state: 0 no usable checkpoint, 1 resume (st, ref_res filled), 2 finished
inline int read_one_state(const char* name, const WorkStatus& want, WorkStatus& st, std::vector<uint64_t>& res) {
    FILE* in = fopen(name, "rb");
    if (!in) return 0;
    int r = 1;
    res.assign(2 * (size_t)want.tpcount, 0);
    if (fread(&st, sizeof(WorkStatus), 1, in) != 1 || fread(res.data(), 16, want.tpcount, in) != want.tpcount) {
        fprintf(stderr, "Cannot parse %s !!!\n", name);
        printf("Cannot parse %s !!!\n", name);
        r = 0;
    } else if (st.tpcount != want.tpcount || st.pmin != want.pmin || st.pmax != want.pmax) {
        fprintf(stderr, "Invalid checkpoint file %s !!!\n", name);
        printf("Invalid checkpoint file %s !!!\n", name);
        r = 0;
    } else if (st.done) {
        r = 2;
    } else if (state_checksum(st, res) != st.state_sum) {
        fprintf(stderr, "Checksum error in %s !!!\n", name);
        printf("Checksum error in %s !!!\n", name);
        r = 0;
    }
    fclose(in);
    return r;
}

inline int read_state(bool& write_a_next, WorkStatus& st, std::vector<uint64_t>& ref_res) {
    WorkStatus a, b;
    std::vector<uint64_t> ra, rb;
    const int ga = read_one_state(STATE_FILENAME_A, st, a, ra);
    if (ga == 2) return 2;
    const int gb = read_one_state(STATE_FILENAME_B, st, b, rb);
    if (gb == 2) return 2;
    if (ga == 1 && (gb != 1 || a.currp > b.currp)) {
        st = a;
        ref_res.swap(ra);
        write_a_next = false;
        return 1;
    }
    if (gb == 1) {
        st = b;
        ref_res.swap(rb);
        write_a_next = true;
        return 1;
    }
    return 0;
}

