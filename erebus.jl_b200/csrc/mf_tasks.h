// mf_tasks.h -- task maps and partial-sum offsets of the triangular solve's
// cooperative levels (inverted pivot blocks), shared by the device solver
// (mfront.cu) and the CPU check of the maps in the test suite.
//
// A cooperative level's forward sweep runs two phases of independent tasks,
// its backward sweep two more; each task streams a run of one row block's
// tiles and writes one 64-entry row product (or a partial of one):
//   F1  pivot row block I < Kt, tiles (I, K), K < I, in chunks of MF_F1_CHUNK;
//   F2  update row block I >= Kt, tiles (I, K), K < Kt, one task per row, or
//       in chunks of MF_F1_CHUNK on levels that chunk long rows;
//   B1  pivot row block K, ring tiles (K, J), J >= Kt, in chunks of
//       MF_RING_CHUNK;
//   B2  pivot row block K, tiles (K, J), J >= K, one task per row, or in
//       chunks of MF_F1_CHUNK on levels that chunk long rows.
// Partial sums of a front live in MfFront::poff + [0, 64 mf_part_slots):
// the B1 ring partials (Kt x ring chunks), the F1 partials of chunks after
// the first (Kt x mf_f1_slots), then one slot per chunk of every row block
// when the front has rows of more than MF_F1_CHUNK tiles.
#pragma once
#include "mf_plan.h"

#ifdef __CUDACC__
#define MF_HD __host__ __device__ __forceinline__
#else
#define MF_HD inline
#endif

namespace erebus {

constexpr int MF_RING_CHUNK = 16;   // ring tiles per B1 task
constexpr int MF_F1_CHUNK = 8;      // tiles per chunk of a pivot row (F1) and of a long row

MF_HD int mf_ring_chunks(int nr) { return (nr + MF_RING_CHUNK - 1) / MF_RING_CHUNK; }

// F1 splits pivot row block I's products over K < I into chunks of
// MF_F1_CHUNK tiles (the root's last row would stream 37 tiles through one
// CTA): chunk 0 stores y_I's gathered entries minus its products, chunks 1..
// store their products as partial sums, and readers of y subtract those in
// chunk order.
MF_HD int mf_f1_chunks(int I) {
    return I <= MF_F1_CHUNK ? 1 : (I + MF_F1_CHUNK - 1) / MF_F1_CHUNK;
}
// F1 tasks of a front: sum over I < Kt of mf_f1_chunks(I), i.e. 1 (I = 0)
// plus sum_{I=1}^{n} ceil(I / 8), n = Kt - 1
MF_HD int mf_f1_tasks(int Kt) {
    if (Kt <= 0) return 0;
    const int n = Kt - 1, q = n / MF_F1_CHUNK, r = n % MF_F1_CHUNK;
    return 1 + MF_F1_CHUNK * q * (q + 1) / 2 + r * (q + 1);
}
// partial-sum slots per pivot row block (the chunks after the first)
MF_HD int mf_f1_slots(int Kt) { return Kt >= 2 ? mf_f1_chunks(Kt - 1) - 1 : 0; }

// chunks of a long row of n tiles (F2, B2)
MF_HD int mf_row_chunks(int n) {
    return n <= MF_F1_CHUNK ? 1 : (n + MF_F1_CHUNK - 1) / MF_F1_CHUNK;
}
// B2 tasks of a front with chunked rows: sum over K < Kt of
// mf_row_chunks(Kt - K), i.e. sum_{m=1}^{Kt} ceil(m / 8)
MF_HD int mf_b2_tasks(int Kt) {
    if (Kt <= 0) return 0;
    const int q = Kt / MF_F1_CHUNK, r = Kt % MF_F1_CHUNK;
    return MF_F1_CHUNK * q * (q + 1) / 2 + r * (q + 1);
}
// partial-sum slots of a front's chunked rows: chunks of every row block
MF_HD long long mf_row_slots(int Kt, int Mt) {
    return Kt > MF_F1_CHUNK ? (long long)Mt * mf_row_chunks(Kt) : 0;
}
// all partial-sum slots of a front (64 doubles each)
MF_HD long long mf_part_slots(int Kt, int Mt) {
    return (long long)Kt * (mf_ring_chunks(Mt - Kt) + mf_f1_slots(Kt)) + mf_row_slots(Kt, Mt);
}

// offset of B1 ring partial ch of pivot row block K
MF_HD long long mf_ring_part(const MfFront &f, int K, int ch) {
    return f.poff + ((long long)K * mf_ring_chunks(f.Mt - f.Kt) + ch) * 64;
}
// offset of pivot row block I's F1 partial ch (>= 1): after the ring partials
MF_HD long long mf_f1_part(const MfFront &f, int I, int ch) {
    return f.poff + (long long)f.Kt * mf_ring_chunks(f.Mt - f.Kt) * 64 +
           ((long long)I * mf_f1_slots(f.Kt) + ch - 1) * 64;
}
// offset of chunk ch of row block I's partial: after the ring and F1 partials
MF_HD long long mf_row_part(const MfFront &f, int I, int ch) {
    return f.poff + (long long)f.Kt * (mf_ring_chunks(f.Mt - f.Kt) + mf_f1_slots(f.Kt)) * 64 +
           ((long long)I * mf_row_chunks(f.Kt) + ch) * 64;
}

// ---- the tasks of a front: counts and decoding of task u ----
// Each decoder gives the row block, the chunk, the first tile's column (k0,
// or the offset i0 from the diagonal for B2) and the number of tiles n.

MF_HD void mf_f1_task(int Kt, int u, int &I, int &ch, int &k0, int &n) {
    (void)Kt;
    I = 0;
    while (u >= mf_f1_chunks(I)) u -= mf_f1_chunks(I++);
    ch = u;
    k0 = ch * MF_F1_CHUNK;
    n = (I < k0 + MF_F1_CHUNK ? I : k0 + MF_F1_CHUNK) - k0;
}

// F2 with nrc chunks per row (1, or mf_row_chunks(Kt) on chunking levels)
MF_HD int mf_f2_tasks(int Kt, int Mt, int nrc) { return (Mt - Kt) * nrc; }
MF_HD void mf_f2_task(int Kt, int nrc, int u, int &I, int &ch, int &k0, int &n) {
    I = Kt + u / nrc;
    ch = u % nrc;
    k0 = ch * MF_F1_CHUNK;
    n = nrc == 1 ? Kt : (MF_F1_CHUNK < Kt - k0 ? MF_F1_CHUNK : Kt - k0);
}

MF_HD int mf_b1_tasks(int Kt, int Mt) { return Kt * mf_ring_chunks(Mt - Kt); }
MF_HD void mf_b1_task(int Kt, int Mt, int u, int &K, int &ch, int &j0, int &n) {
    const int nch = mf_ring_chunks(Mt - Kt);
    K = u / nch;
    ch = u % nch;
    j0 = Kt + ch * MF_RING_CHUNK;
    n = MF_RING_CHUNK < Mt - j0 ? MF_RING_CHUNK : Mt - j0;
}

// B2, with chunked long rows or one task per row; nrc is the row's chunks
MF_HD int mf_b2_count(int Kt, bool chunked) { return chunked ? mf_b2_tasks(Kt) : Kt; }
MF_HD void mf_b2_task(int Kt, bool chunked, int u, int &K, int &ch, int &nrc, int &i0,
                      int &n) {
    K = 0;
    if (chunked) {
        while (u >= mf_row_chunks(Kt - K)) u -= mf_row_chunks(Kt - K++);
    } else {
        K = u;
        u = 0;
    }
    ch = u;
    const int m = Kt - K;
    nrc = chunked ? mf_row_chunks(m) : 1;
    i0 = ch * MF_F1_CHUNK;
    n = nrc == 1 ? m : (MF_F1_CHUNK < m - i0 ? MF_F1_CHUNK : m - i0);
}

}  // namespace erebus

#undef MF_HD
