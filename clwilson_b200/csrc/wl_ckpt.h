// wl_ckpt.h -- checkpoint files of the clwilson program in the reference's
// format (cl_wilson.h:22-25, cl_wilson.cpp:110-288): the workStatus header,
// then one (s0, s1) pair per test prime, the running products in the
// reference's Montgomery form (R = 2^64 mod p^2, base-p digits), and the
// additive state_sum; two files written alternately.
//
// Which files the two programs can share.  Below 2^32 both programs multiply
// in exact primes.  From 2^32 on the reference multiplies in every base-2
// strong probable prime that passes its 7..113 presieve (getsegprps.cl:211-293)
// and divides the pseudoprimes among them (prps.dat) out of each row at the
// very end, whatever its checkpoint's currp (cl_wilson.cpp:709-726); this
// engine's columns above 2^32 are exact primes.  So a checkpoint whose columns
// stop at currp <= 2^32 means the same thing to both programs, and one past
// 2^32 does not: a reference file past 2^32 holds pseudoprime factors this
// program never removes, and a file of this program past 2^32 lacks factors
// that the reference would divide out.  Therefore:
//   * checkpoints with currp <= 2^32, and finished ones, use the reference's
//     names stateA.ckp / stateB.ckp;
//   * checkpoints past 2^32 go to this program's own stateA.b200.ckp /
//     stateB.b200.ckp, which the reference never reads;
//   * a reference-named file past 2^32 that is not finished is refused
//     (read_state returns 3) instead of being resumed with a wrong product.
// Host code only (no CUDA).
#pragma once
#include <cstdint>
#include <cstdio>
#include <vector>

static const char* const STATE_FILENAME_A = "stateA.ckp";
static const char* const STATE_FILENAME_B = "stateB.ckp";
static const char* const OWN_STATE_FILENAME_A = "stateA.b200.ckp";
static const char* const OWN_STATE_FILENAME_B = "stateB.b200.ckp";
// Largest currp whose running products mean the same to the reference and to
// this program (columns q < currp, all below 2^32).
static const uint64_t CKPT_SHARED_CURRP = 1ull << 32;

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

// write_state: the header then tpcount residue pairs, alternating A and B; the
// reference's file names up to currp = 2^32 and for a finished workunit, this
// program's own names past 2^32
inline void write_state(bool& write_a_next, WorkStatus& st, const std::vector<uint64_t>& ref_res) {
    st.state_sum = state_checksum(st, ref_res);
    const bool shared = st.done || st.currp <= CKPT_SHARED_CURRP;
    const char* name = write_a_next ? (shared ? STATE_FILENAME_A : OWN_STATE_FILENAME_A)
                                    : (shared ? STATE_FILENAME_B : OWN_STATE_FILENAME_B);
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

// read_state: 0 no usable checkpoint, 1 resume (st, ref_res filled), 2
// finished, 3 refused (a reference-named file past 2^32, see the top)
inline int read_state(bool& write_a_next, WorkStatus& st, std::vector<uint64_t>& ref_res) {
    const char* names[4] = { STATE_FILENAME_A, STATE_FILENAME_B, OWN_STATE_FILENAME_A, OWN_STATE_FILENAME_B };
    WorkStatus got[4];
    std::vector<uint64_t> res[4];
    int status[4];
    for (int i = 0; i < 4; ++i) {
        status[i] = read_one_state(names[i], st, got[i], res[i]);
        if (status[i] == 2) return 2;
    }
    for (int i = 0; i < 2; ++i) {
        if (status[i] == 1 && got[i].currp > CKPT_SHARED_CURRP) {
            fprintf(stderr, "Checkpoint %s stops at P %llu, past 2^32, where its running products hold base-2 "
                    "pseudoprime factors that only the reference program removes; finish this range with that "
                    "program, or delete %s and %s to start over.\n", names[i], (unsigned long long)got[i].currp,
                    STATE_FILENAME_A, STATE_FILENAME_B);
            printf("Checkpoint %s stops at P %llu, past 2^32, where its running products hold base-2 "
                   "pseudoprime factors that only the reference program removes; finish this range with that "
                   "program, or delete %s and %s to start over.\n", names[i], (unsigned long long)got[i].currp,
                   STATE_FILENAME_A, STATE_FILENAME_B);
            return 3;
        }
    }
    int best = -1;
    for (int i = 0; i < 4; ++i)
        if (status[i] == 1 && (best < 0 || got[i].currp > got[best].currp)) best = i;
    if (best < 0) return 0;
    st = got[best];
    ref_res.swap(res[best]);
    write_a_next = (best % 2) == 1;   // the other file of the pair is written next
    return 1;
}
