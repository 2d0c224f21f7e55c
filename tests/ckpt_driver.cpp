// Test driver for clwilson_b200/csrc/wl_ckpt.h (the checkpoint format), used
// by tests/test_checkpoint_format.py.  Commands:
//   conv p s0 s1                       to_reference, then from_reference
//   write A|B pmin pmax currp trickle totalcount done r0 r1 ...
//   read pmin pmax tpcount             read_state: status, currp, next file, residues
#include <cinttypes>
#include <cstdlib>
#include <cstring>
#include "wl_ckpt.h"

static uint64_t u(const char* s) { return strtoull(s, nullptr, 0); }

int main(int argc, char** argv) {
    if (argc >= 5 && !strcmp(argv[1], "conv")) {
        uint64_t r0, r1, s0, s1;
        to_reference(u(argv[2]), u(argv[3]), u(argv[4]), &r0, &r1);
        from_reference(u(argv[2]), r0, r1, &s0, &s1);
        printf("%" PRIu64 " %" PRIu64 " %" PRIu64 " %" PRIu64 "\n", r0, r1, s0, s1);
        return 0;
    }
    if (argc >= 9 && !strcmp(argv[1], "write")) {
        bool a_next = argv[2][0] == 'A';
        WorkStatus st;
        memset(&st, 0, sizeof(st));
        st.pmin = u(argv[3]); st.pmax = u(argv[4]); st.currp = u(argv[5]); st.trickle = u(argv[6]);
        st.totalcount = u(argv[7]); st.done = (uint32_t)u(argv[8]);
        std::vector<uint64_t> res;
        for (int i = 9; i < argc; ++i) res.push_back(u(argv[i]));
        st.tpcount = (uint32_t)(res.size() / 2);
        write_state(a_next, st, res);
        printf("next %s\n", a_next ? "A" : "B");
        return 0;
    }
    if (argc >= 5 && !strcmp(argv[1], "read")) {
        WorkStatus st;
        memset(&st, 0, sizeof(st));
        st.pmin = u(argv[2]); st.pmax = u(argv[3]); st.tpcount = (uint32_t)u(argv[4]);
        std::vector<uint64_t> res;
        bool a_next = true;
        const int r = read_state(a_next, st, res);
        printf("status %d currp %" PRIu64 " next %s", r, st.currp, a_next ? "A" : "B");
        for (size_t i = 0; r == 1 && i < res.size(); ++i) printf(" %" PRIu64, res[i]);
        printf("\n");
        return 0;
    }
    return 2;
}
