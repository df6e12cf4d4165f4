// Internal constants and small helpers shared by the host-side code of
// libcmscan_gpu.so.  State / node codes follow src/constants.rs:9-93 of the
// reference (they are the on-disk and in-memory codes of Infernal CMs).
#pragma once
#include <cmath>
#include <cstdint>

namespace cmx {

// state types (src/constants.rs:9-18)
constexpr int D_ST = 0, MP_ST = 1, ML_ST = 2, MR_ST = 3, IL_ST = 4, IR_ST = 5,
              S_ST = 6, E_ST = 7, B_ST = 8, EL_ST = 9;
// node types (src/constants.rs:24-31)
constexpr int BIF_ND = 0, MATP_ND = 1, MATL_ND = 2, MATR_ND = 3, BEGL_ND = 4,
              BEGR_ND = 5, ROOT_ND = 6, END_ND = 7;
// unique state ids used by the scanners (src/constants.rs:46-81)
constexpr int ROOT_S = 0, BEGL_S = 3, BEGR_S = 4, MATP_IR = 11;

constexpr int K = 4;          // canonical alphabet
constexpr int KP = 18;        // digital alphabet incl. degeneracies
constexpr int MAXC = 6;       // CM_MAXCONNECT
constexpr int ESC = 324;      // per-state emission row (18*18)
constexpr int INFTY = 987654321;
constexpr double INTSCALE = 1000.0;
constexpr float IMPOSSIBLE = -1.0e36f;
constexpr int LOGSUM_TBL = 23000;

inline int state_delta(int st) {
    return st == MP_ST ? 2 : (st == ML_ST || st == MR_ST || st == IL_ST || st == IR_ST) ? 1 : 0;
}
inline int state_right_delta(int st) {
    return (st == MP_ST || st == MR_ST || st == IR_ST) ? 1 : 0;
}
inline bool right_emitter(int st) { return state_right_delta(st) > 0; }

// IUPAC degeneracy of the digital RNA alphabet "ACGU-RYMKSWHBVDN*~"
// (src/cm.rs:24-43).  bit l set when code x includes canonical residue l.
constexpr uint8_t DEGEN_BITS[KP] = {0x1, 0x2, 0x4, 0x8, 0x0, 0x5, 0xA, 0x3, 0xC,
                                    0x6, 0x9, 0xB, 0xE, 0x7, 0xD, 0xF, 0x0, 0x0};
inline bool degen(int x, int l) { return (DEGEN_BITS[x] >> l) & 1; }
inline int ndegen(int x) {
    int c = 0;
    for (int l = 0; l < K; l++) c += degen(x, l);
    return c;
}
inline bool is_residue(int x) { return x < K || (x > K && x < KP - 2); }
// esl_abc_FCount fraction (src/cm.rs:72-79)
inline float fcount_frac(int x, int l) {
    return degen(x, l) ? 1.0f / (float)ndegen(x) : 0.0f;
}

// sreLOG2: x > 0 ? ln(x) * 1.44269504 : IMPOSSIBLE (src/cm_nohmm.rs:46-53)
inline double sre_log2(double x) { return x > 0.0 ? std::log(x) * 1.44269504 : -1.0e36; }

}  // namespace cmx
