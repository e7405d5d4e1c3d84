// Per-warp column reduction of element-pair blocks (mixed P1 kernels).
//
// The 32 lanes of a warp are 32 consecutive trial elements; their 96 local
// dof slots (lane, j) fall on far fewer distinct dofs -- ~27 on a mesh
// numbered with locality such as the refined spheres -- because neighbouring
// elements share vertices.  Instead of one FP64 atomic per slot and block
// row, the lanes stage their block values in shared memory, grouped by
// column (distinct trial dof), and after __syncwarp each column's slots are
// summed by one lane and added to the matrix once: ~3.5x fewer L2 atomics for
// the same FP64 values.  The columns come from a 128-entry hash table per
// warp (32-bit shared-memory CAS, linear probing); a column's slots take
// consecutive staging positions (offset of the column + rank of the slot).
#pragma once

#include "common.cuh"

namespace bc {

constexpr int WC_SLOTS = 96;   // 32 lanes x 3 local dofs
constexpr int WC_TABLE = 128;  // hash table entries (> WC_SLOTS, a power of 2)

struct WarpColumns {
    int col[WC_SLOTS];        // column -> dof
    int start[WC_SLOTS + 1];  // column -> first staging position; start[ncols] = staged slots
    int ncols;
};

// Columns of the warp's slots; every lane of the warp calls it with its 3 dofs (negative: no slot).
// Returns each slot's staging position in pos[j] (-1 for no slot).  scratch: 2 x WC_TABLE ints of
// the warp's own (the staging array, which is written only after this returns).
__device__ __forceinline__ void wc_build(WarpColumns &wc, int *scratch, const int dof[3], int pos[3]) {
    const unsigned lane = threadIdx.x & 31u;
    struct Table {
        int key[WC_TABLE];  // dof, or -1 (empty)
        int off[WC_TABLE];  // slots with that dof, then the column's first staging position
    } &wt = *reinterpret_cast<Table *>(scratch);
#pragma unroll
    for (int e = 0; e < WC_TABLE / 32; ++e) {
        wt.key[lane + 32 * e] = -1;
        wt.off[lane + 32 * e] = 0;
    }
    __syncwarp();
    int h[3], rank[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        h[j] = -1;
        rank[j] = 0;
        if (dof[j] < 0) continue;
        int t = (int)(((unsigned)dof[j] * 2654435761u) >> 25);  // top 7 bits: 0 .. 127
        // at most 96 distinct keys in 128 entries: an empty or matching entry is always found
        for (int probe = 0; probe < WC_TABLE; ++probe) {
            const int old = atomicCAS(&wt.key[t], -1, dof[j]);
            if (old == -1 || old == dof[j]) break;
            t = (t + 1) & (WC_TABLE - 1);
        }
        h[j] = t;
        rank[j] = atomicAdd(&wt.off[t], 1);
    }
    __syncwarp();
    // columns in table order: each lane takes 4 consecutive entries, a warp scan gives the offsets
    int cnt[4], used = 0, total = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        cnt[e] = wt.off[4 * lane + e];
        used += cnt[e] > 0;
        total += cnt[e];
    }
    int used_incl = used, total_incl = total;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, used_incl, d), s = __shfl_up_sync(0xffffffffu, total_incl, d);
        if ((int)lane >= d) {
            used_incl += u;
            total_incl += s;
        }
    }
    int c = used_incl - used, o = total_incl - total;
    __syncwarp();
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        if (cnt[e] == 0) continue;
        wc.col[c] = wt.key[4 * lane + e];
        wc.start[c] = o;
        wt.off[4 * lane + e] = o;
        ++c;
        o += cnt[e];
    }
    if (lane == 31) {
        wc.ncols = used_incl;
        wc.start[used_incl] = total_incl;
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 3; ++j) pos[j] = h[j] < 0 ? -1 : wt.off[h[j]] + rank[j];
    __syncwarp();
}

}  // namespace bc
