// Nearest-parcel search and merging on the device with the single-rank
// semantics of the reference (parcel_nearest.f90, parcel_merge.f90,
// parcel_container.f90:413-458).  Index decisions are bit-exact with the
// oracle on identical inputs:
//   * cell binning and nearest-grid-point rounding reproduce int / nint
//     (parcel_nearest.f90:196-226, 675-699);
//   * the boundary copies that stand in for the MPI neighbour exchange are
//     appended in the reference's receive order (parcel_nearest.f90:1466-1621,
//     mpi_tags.f90:13-31) and binned after the local parcels, so every cell
//     lists its parcels in ascending index order (stable radix sort);
//   * distances use non-contracted arithmetic and the same strict '<' / '>'
//     comparisons (parcel_nearest.f90:717-723, 901);
//   * resolve_tree stage 1 is four parallel passes per iteration; the
//     order-dependent stage-2 loop (parcel_nearest.f90:1220-1311) is resolved
//     with a fixed-point iteration along its dependency chains;
//   * each merge group is reduced by one thread in m order, so the merged
//     attributes round like the reference's sequential loop.
#include "ctx.hpp"
#include "eigen.cuh"

#include <cub/cub.cuh>
#include <cstring>
#include <vector>
#include <algorithm>

namespace epic {

constexpr int MB = 256;

static int mgrid(long long n) {
    long long b = (n + MB - 1) / MB;
    return (int)std::max<long long>(1, std::min<long long>(b, 148LL * 32));
}

#define MLOOP(n) for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); \
                      i += (long long)gridDim.x * blockDim.x)

struct Box {
    int hs1, hs2;          // box%halo_size(1:2) = nx+3, ny+3
    long long hncell;      // (nx+3)(ny+3)(nz+2)
};

// parcel_to_local_cell_index incl. handle_periodic_edge_parcels
// (parcel_nearest.f90:166-226); may shift x, y by one period.
EPIC_DEV int bin_cell(const Params& P, const Box& B, double& x, double& y, double z, unsigned* err) {
    int gx = (int)floor(ExactOps::mul(ExactOps::sub(x, P.lower[0]), P.dxi[0]));
    int gy = (int)floor(ExactOps::mul(ExactOps::sub(y, P.lower[1]), P.dxi[1]));
    if (gx < -1) x = ExactOps::add(x, P.extent[0]);
    if (gx > P.nx) x = ExactOps::sub(x, P.extent[0]);
    if (gy < -1) y = ExactOps::add(y, P.extent[1]);
    if (gy > P.ny) y = ExactOps::sub(y, P.extent[1]);
    int ix = (int)ExactOps::mul(P.dxi[0], ExactOps::sub(x, P.halo_lower[0]));
    int iy = (int)ExactOps::mul(P.dxi[1], ExactOps::sub(y, P.halo_lower[1]));
    int iz = min((int)ExactOps::mul(P.dxi[2], ExactOps::sub(z, P.lower[2])), P.nz - 1);
    long long ijk = (long long)ix + (long long)B.hs1 * iy + (long long)B.hs1 * B.hs2 * iz;
    if (ijk < 0 || ijk >= B.hncell || ix < 0 || iy < 0) {
        set_err(err, ERRB_CELL);
        return 0;
    }
    return (int)ijk;
}

EPIC_DEV int nint_d(double v) { return (int)round(v); }

// send buffer bits (mpi_tags.f90:3-11): 1 N, 2 S, 3 W, 4 E, 5 NW, 6 NE, 7 SW, 8 SE
// locate_parcel_in_boundary_cell (parcel_nearest.f90:1384-1460)
EPIC_DEV unsigned boundary_bits(const Params& P, double x, double y) {
    int ix = nint_d(ExactOps::mul(P.dxi[0], ExactOps::sub(x, P.lower[0])));
    int iy = nint_d(ExactOps::mul(P.dxi[1], ExactOps::sub(y, P.lower[1])));
    unsigned b = 0;
    if (ix == 0) {
        if (iy == 0) b |= 1u << 7;
        else if (iy == P.ny) b |= 1u << 5;
        b |= 1u << 3;
    }
    if (ix == P.nx) {
        if (iy == 0) b |= 1u << 8;
        else if (iy == P.ny) b |= 1u << 6;
        b |= 1u << 4;
    }
    if (iy == 0) b |= 1u << 2;
    if (iy == P.ny) b |= 1u << 1;
    return b;
}

// M1: bin the local parcels, flag small ones and their boundary buffers.
__global__ void k_bin_locals(Params P, Box B, PView pv, int N, int* cell, int* small, unsigned* bits,
                             unsigned* err) {
    MLOOP(N) {
        double x = pv.get(A_X, i), y = pv.get(A_Y, i), z = pv.get(A_Z, i);
        double x0 = x, y0 = y;
        cell[i] = bin_cell(P, B, x, y, z, err);
        if (x != x0) pv.set(A_X, i, x);
        if (y != y0) pv.set(A_Y, i, y);
        int s = pv.get(A_VOL, i) < P.vmin;
        small[i] = s;
        bits[i] = s ? boundary_bits(P, x, y) : 0u;
    }
}

// receive slot r (1..8) holds send buffer SEND_NEIGHBOUR_TAG^-1(r)
__constant__ int c_slot_buf[9] = {0, 2, 1, 4, 3, 8, 7, 6, 5};

// M3 flags in copy order: F[(r-1)*nls + m] = small m is copied into slot r
__global__ void k_copy_flags(const int* Ls, int nls, const unsigned* bits, int* F) {
    MLOOP((long long)8 * nls) {
        int r = (int)(i / nls) + 1;
        int m = (int)(i - (long long)(r - 1) * nls);
        F[i] = (bits[Ls[m]] >> c_slot_buf[r]) & 1u;
    }
}

struct CopyArgs {
    double* cx;
    double* cy;
    double* cz;
    int* pid;      // original parcel (0-based)
    int* mid;      // merge index of the original (0-based in the local small list)
};

// M4: materialise the copies with apply_periodic_shift (parcel_nearest.f90:630-668)
__global__ void k_make_copies(Params P, Box B, PView pv, const int* Ls, int nls, const int* F, const int* off,
                              CopyArgs C, int* cell_copies, int* copyidx, unsigned* err) {
    MLOOP((long long)8 * nls) {
        if (!F[i]) continue;
        int r = (int)(i / nls) + 1;
        int m = (int)(i - (long long)(r - 1) * nls);
        int q = off[i];
        int n = Ls[m];
        double x = pv.get(A_X, n), y = pv.get(A_Y, n), z = pv.get(A_Z, n);
        int ix = nint_d(ExactOps::mul(P.dxi[0], ExactOps::sub(x, P.lower[0])));
        int iy = nint_d(ExactOps::mul(P.dxi[1], ExactOps::sub(y, P.lower[1])));
        bool xe = (ix <= 0) || (ix >= P.nx), ye = (iy <= 0) || (iy >= P.ny);
        double Lx = P.extent[0], Ly = P.extent[1];
        switch (r) {
            case 1: if (ye) y = ExactOps::add(y, Ly); break;
            case 2: if (ye) y = ExactOps::sub(y, Ly); break;
            case 3: if (xe) x = ExactOps::sub(x, Lx); break;
            case 4: if (xe) x = ExactOps::add(x, Lx); break;
            case 5: if (xe) x = ExactOps::sub(x, Lx); if (ye) y = ExactOps::add(y, Ly); break;
            case 6: if (xe) x = ExactOps::add(x, Lx); if (ye) y = ExactOps::add(y, Ly); break;
            case 7: if (xe) x = ExactOps::sub(x, Lx); if (ye) y = ExactOps::sub(y, Ly); break;
            case 8: if (xe) x = ExactOps::add(x, Lx); if (ye) y = ExactOps::sub(y, Ly); break;
        }
        cell_copies[q] = bin_cell(P, B, x, y, z, err);
        C.cx[q] = x; C.cy[q] = y; C.cz[q] = z;
        C.pid[q] = n;
        C.mid[q] = m;
        copyidx[(long long)(c_slot_buf[r] - 1) * nls + m] = q;
    }
}

__global__ void k_iota(int* v, long long n) { MLOOP(n) v[i] = (int)i; }
__global__ void k_iota_from(int* v, long long n, int first) { MLOOP(n) v[i] = first + (int)i; }

// Box-ordered store (Ctx::rank): per-parcel values in container order
// (ord[r] = slot of container index r).
__global__ void k_by_rank(const int* ord, const int* a, long long n, int* ar) { MLOOP(n) ar[i] = a[ord[i]]; }
// the local entries of the binning sort in container order: keys cell, values slot
__global__ void k_rank_cells(const int* ord, const int* cell0, long long n, int* cell, int* vals) {
    MLOOP(n) {
        const int s = ord[i];
        cell[i] = cell0[s];
        vals[i] = s;
    }
}
__global__ void k_pairs_rank(const int* rank, const int* ism, const int* icl, int nm, int* ri, int* rc) {
    MLOOP(nm) {
        ri[i] = rank[ism[i]];
        rc[i] = rank[icl[i]];
    }
}
// parcel_delete in container indices (parcel_container.f90:413-458): flags of
// the deleted indices below newN (holes) and of the kept ones from newN up
// (sources)
__global__ void k_del_rank_flags(const int* ord, const char* del, int N, int newN, int* hole, int* src) {
    MLOOP(N) {
        const int d = del[ord[i]];
        hole[i] = (i < newN) && d;
        src[i] = (i >= newN) && !d;
    }
}
// the i-th hole (ascending) takes the kept parcel with the i-th largest index
__global__ void k_rerank(const int* ord, const int* holes, const int* srcs, int nh, int* rank) {
    MLOOP(nh) rank[ord[srcs[nh - 1 - i]]] = holes[i];
}

// M6: cell ranges of the sorted (cell, index) list
__global__ void k_cell_ranges(const int* keys, long long nt, int* cstart, int* cend) {
    MLOOP(nt) {
        int k = keys[i];
        if (i == 0 || keys[i - 1] != k) cstart[k] = (int)i;
        if (i == nt - 1 || keys[i + 1] != k) cend[k] = (int)i + 1;
    }
}

EPIC_DEV void entry_pos(const PView& pv, const CopyArgs& C, int N, int j, double& x, double& y, double& z) {
    if (j < N) { x = pv.get(A_X, j); y = pv.get(A_Y, j); z = pv.get(A_Z, j); }
    else { x = C.cx[j - N]; y = C.cy[j - N]; z = C.cz[j - N]; }
}

// Positions of the sorted entries in cell order, with the entry index as the
// bit pattern of w: the search then streams through a cell's candidates
// (one 32-byte record each) instead of gathering an index and three
// attributes per candidate from the parcel store.
__global__ void k_sorted_pos(PView pv, CopyArgs C, int N, const int* sorted_idx, long long nt, double4* sp) {
    MLOOP(nt) {
        const int j = sorted_idx[i];
        double x, y, z;
        entry_pos(pv, C, N, j, x, y, z);
        sp[i] = make_double4(x, y, z, __longlong_as_double((long long)j));
    }
}

// Cells of the small entries (locals m < nls, then the copies), for the
// search order.
__global__ void k_small_keys(const int* Ls, int nls, int ncp, const int* cell0, const int* cell_copies, int* keys,
                             int* vals) {
    MLOOP((long long)nls + ncp) {
        keys[i] = i < nls ? cell0[Ls[i]] : cell_copies[i - nls];
        vals[i] = (int)i;
    }
}

// M8: find_closest_parcel_locally (parcel_nearest.f90:675-747) for every small
// entry m (locals 0..nls-1, then copies).  sp: the sorted entries' positions
// (k_sorted_pos), or null to read them through sorted_idx.  order: the small
// entries by cell, so that the lanes of a warp search neighbouring cells (the
// same candidates, similar trip counts), or null; each entry's result does
// not depend on the order.
__global__ void k_search(Params P, Box B, PView pv, CopyArgs C, int N, const int* Ls, int nls, int ncp,
                         const int* sorted_idx, const double4* sp, const int* order, const int* cstart,
                         const int* cend, int* iclo, double* dclo) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)nls + ncp;
         t += (long long)gridDim.x * blockDim.x) {
        const long long i = order ? order[t] : t;
        int is = i < nls ? Ls[i] : N + (int)(i - nls);
        double xs, ys, zs;
        entry_pos(pv, C, N, is, xs, ys, zs);
        int ix0 = nint_d(ExactOps::mul(P.dxi[0], ExactOps::sub(xs, P.halo_lower[0])));
        int iy0 = nint_d(ExactOps::mul(P.dxi[1], ExactOps::sub(ys, P.halo_lower[1])));
        int iz0 = nint_d(ExactOps::mul(P.dxi[2], ExactOps::sub(zs, P.lower[2])));
        double dsqmin = ExactOps::add(ExactOps::add(ExactOps::mul(P.extent[0], P.extent[0]),
                                                    ExactOps::mul(P.extent[1], P.extent[1])),
                                      ExactOps::mul(P.extent[2], P.extent[2]));
        int ic = -1;
        for (int iz = max(0, iz0 - 1); iz <= min(P.nz - 1, iz0); ++iz)
            for (int iy = max(0, iy0 - 1); iy <= min(P.ny + 1, iy0); ++iy)
                for (int ix = max(0, ix0 - 1); ix <= min(P.nx + 1, ix0); ++ix) {
                    long long ijk = (long long)ix + (long long)B.hs1 * iy + (long long)B.hs1 * B.hs2 * iz;
                    int k1 = cstart[ijk], k2 = cend[ijk];
                    for (int k = k1; k < k2; ++k) {
                        int nn;
                        double xn, yn, zn;
                        if (sp) {
                            const double4 e = sp[k];
                            nn = (int)__double_as_longlong(e.w);
                            xn = e.x; yn = e.y; zn = e.z;
                        } else {
                            nn = sorted_idx[k];
                            if (nn != is) entry_pos(pv, C, N, nn, xn, yn, zn);
                        }
                        if (nn == is) continue;
                        double delz = ExactOps::sub(zn, zs);
                        if (ExactOps::mul(delz, delz) < dsqmin) {
                            double delx = ExactOps::sub(xn, xs);
                            double dely = ExactOps::sub(yn, ys);
                            double dsq = ExactOps::add(ExactOps::add(ExactOps::mul(delx, delx), ExactOps::mul(dely, dely)),
                                                       ExactOps::mul(delz, delz));
                            if (dsq < dsqmin) { dsqmin = dsq; ic = nn; }
                        }
                    }
                }
        // update_remote_indices (parcel_nearest.f90:751-794)
        if (is >= N && ic >= N) dsqmin = 1.7976931348623157e308;
        else if (ic >= N) ic = C.pid[ic - N];
        iclo[i] = ic;
        dclo[i] = dsqmin;
    }
}

// M10: find_closest_parcel_globally (parcel_nearest.f90:804-930): copy results
// return to the originals in send-buffer order 1..8, strict '>'.
__global__ void k_globally(int nls, const int* copyidx, int* iclo, double* dclo, unsigned* err) {
    MLOOP(nls) {
        double d = dclo[i];
        int c = iclo[i];
        for (int k = 0; k < 8; ++k) {
            int q = copyidx[(long long)k * nls + i];
            if (q < 0) continue;
            int mc = nls + q;
            if (d > dclo[mc]) { d = dclo[mc]; c = iclo[mc]; }
        }
        dclo[i] = d;
        iclo[i] = c;
        if (c < 0) set_err(err, ERRB_NO_NEIGHBOUR);
    }
}

// resolve_tree stage 1 (parcel_nearest.f90:953-1154), one pass per kernel
__global__ void k_tree_a(const int* Ls, const int* iclo, int nls, char* merged, char* leaf, char* avail) {
    MLOOP(nls) {
        int is = Ls[i];
        if (!merged[is]) { leaf[is] = 1; avail[iclo[i]] = 1; }
    }
}
__global__ void k_tree_b(const int* Ls, const int* iclo, int nls, const char* merged, char* leaf) {
    MLOOP(nls) {
        if (!merged[Ls[i]]) leaf[iclo[i]] = 0;
    }
}
__global__ void k_tree_c(const int* Ls, const int* iclo, int nls, const char* merged, const char* leaf, char* avail) {
    MLOOP(nls) {
        int is = Ls[i];
        if (!merged[is] && !leaf[is]) avail[iclo[i]] = 0;
    }
}
__global__ void k_tree_d(const int* Ls, const int* iclo, int nls, char* merged, const char* leaf,
                         const char* avail, int* cont) {
    MLOOP(nls) {
        int is = Ls[i];
        if (!merged[is]) {
            int ic = iclo[i];
            if (leaf[is] && avail[ic]) {
                *cont = 1;
                merged[is] = 1;
                merged[ic] = 1;
            }
        }
    }
}

// stage 2 (parcel_nearest.f90:1158-1377).  status: 0 n/a, 1 unknown, 2 merge
// (helper true), 3 isolated dual link.
__global__ void k_tree_e(const int* Ls, const int* iclo, int nls, const char* merged, const char* leaf, char* avail) {
    MLOOP(nls) {
        int is = Ls[i];
        if (!merged[is] && leaf[is]) avail[iclo[i]] = 1;
    }
}
__global__ void k_tree_f_init(const int* Ls, const int* iclo, int nls, const char* merged, const char* leaf,
                              const char* avail, char* dom, char* status, unsigned* err) {
    MLOOP(nls) {
        int is = Ls[i], ic = iclo[i];
        char d = 0, s = 0;
        if (merged[is] && leaf[is]) {
            d = 1;
            if (leaf[ic]) set_err(err, ERRB_TREE);
        } else if (!merged[is]) {
            if (leaf[is]) d = 1;
            else if (!avail[is]) s = 1;
        }
        dom[i] = d;
        status[i] = s;
    }
}
__global__ void k_tree_f_round(const int* iclo, int nls, const int* minv, const char* avail, char* status,
                               int* unknown) {
    MLOOP(nls) {
        if (status[i] != 1) continue;
        int ic = iclo[i];
        char s;
        if (avail[ic]) {
            s = 2;
        } else {
            int mp = minv[ic];
            if (mp < 0 || mp >= (int)i || status[mp] == 0) s = 3;
            else if (status[mp] == 3) s = 2;
            else if (status[mp] == 2) s = 3;
            else { *unknown = 1; continue; }
        }
        status[i] = s;
    }
}
__global__ void k_tree_f_apply(const int* Ls, int nls, const char* status, char* avail, char* dom) {
    MLOOP(nls) {
        if (status[i] == 3) avail[Ls[i]] = 1;
        if (status[i] == 2) dom[i] = 1;
    }
}
__global__ void k_tree_g(const int* iclo, int nls, const char* status, const char* avail, char* dom) {
    MLOOP(nls) {
        if (!dom[i] && status[i] == 3 && avail[iclo[i]]) dom[i] = 1;
    }
}

__global__ void k_pack_pairs(const int* Ls, const int* iclo, int nls, const char* dom, const int* pos,
                             int* ism, int* icl) {
    MLOOP(nls) {
        if (dom[i]) {
            ism[pos[i]] = Ls[i];
            icl[pos[i]] = iclo[i];
        }
    }
}
__global__ void k_char_to_int(const char* a, int* b, long long n) { MLOOP(n) b[i] = a[i]; }
__global__ void k_set_minv(const int* Ls, int nls, int* minv) { MLOOP(nls) minv[Ls[i]] = (int)i; }

__global__ void k_big_close(PView pv, const int* icl, int nm, double vmin, unsigned long long* cnt) {
    unsigned long long local = 0;
    MLOOP(nm) local += pv.get(A_VOL, icl[i]) > vmin;
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffff, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(cnt, local);
}

// group heads of the ic-sorted merge list
__global__ void k_group_heads(const int* keys, int nm, int* head) {
    MLOOP(nm) head[i] = (i == 0 || keys[i - 1] != keys[i]) ? 1 : 0;
}

EPIC_DEV double pdelta(double d, double L, double Li) {
    return d - L * (double)nint_d(d * Li);
}

// The label draw of the merge (parcel_merge.f90:196, random_number): U[0, 1)
// from a counter-based SplitMix64 keyed by (label_seed, merge call, merge
// index m), the same in the oracle.
EPIC_DEV unsigned long long label_mix(unsigned long long x) {
    unsigned long long z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
EPIC_DEV double label_draw(int seed, long long call, long long m) {
    const unsigned long long key = ((unsigned long long)(unsigned)seed * 0x9E3779B97F4A7C15ull) ^
                                   ((((unsigned long long)call << 32) + (unsigned long long)m) * 16ull + 15ull);
    return (double)(label_mix(label_mix(key)) >> 11) * (1.0 / 9007199254740992.0);
}

struct MergeLabels {
    long long* label;   // null: labels off
    double* dil;
    int seed;
    long long call;
};

// do_group_merge + geometric_merge for one group (parcel_merge.f90:118-361)
__global__ void k_group_merge(Params P, PView pv, const int* gstart, int ng, int nm, const int* skeys,
                              const int* svals, const int* ism, MergeLabels L, unsigned* err) {
    MLOOP(ng) {
        int s0 = gstart[i];
        int s1 = (i + 1 < ng) ? gstart[i + 1] : nm;
        int ic = skeys[s0];
        double vic = pv.get(A_VOL, ic);
        double xic = pv.get(A_X, ic), yic = pv.get(A_Y, ic), zic = pv.get(A_Z, ic);
        double vm = vic, x0 = xic, y0 = yic;
        double pm0 = 0.0, pm1 = 0.0, pm2 = vic * zic;
        double bm = vic * pv.get(A_BUOY, ic), hm = vic * pv.get(A_HUM, ic);
        double wm[3] = {vic * pv.get(A_VX, ic), vic * pv.get(A_VY, ic), vic * pv.get(A_VZ, ic)};
        long long labm = L.label ? L.label[ic] : 0;
        double dilm = L.label ? L.dil[ic] : 0.0;
        for (int q = s0; q < s1; ++q) {
            int is = ism[svals[q]];
            double p[3] = {pv.get(A_X, is), pv.get(A_Y, is), pv.get(A_Z, is)};
            // apply_periodic_bc on the small parcel (parcel_merge.f90:143)
            p[0] = p[0] - P.extent[0] * (double)(int)((p[0] - P.center[0]) * P.hli[0]);
            p[1] = p[1] - P.extent[1] * (double)(int)((p[1] - P.center[1]) * P.hli[1]);
            pv.set(A_X, is, p[0]);
            pv.set(A_Y, is, p[1]);
            double v = pv.get(A_VOL, is);
            if (L.label) {
                // parcel_merge.f90:193-203, in m order within the group
                const double rn = label_draw(L.seed, L.call, svals[q]);
                if (rn * (vm + v) < vm) {
                    dilm = dilm + log(vm / (vm + v));
                } else {
                    labm = L.label[is];
                    dilm = L.dil[is] + log(v / (vm + v));
                }
            }
            vm = vm + v;
            double dx = pdelta(p[0] - x0, P.extent[0], P.extenti[0]);
            double dy = pdelta(p[1] - y0, P.extent[1], P.extenti[1]);
            pm0 = pm0 + v * dx;
            pm1 = pm1 + v * dy;
            pm2 = pm2 + v * p[2];
            bm = bm + v * pv.get(A_BUOY, is);
            hm = hm + v * pv.get(A_HUM, is);
            wm[0] = wm[0] + v * pv.get(A_VX, is);
            wm[1] = wm[1] + v * pv.get(A_VY, is);
            wm[2] = wm[2] + v * pv.get(A_VZ, is);
        }
        double vmerge = 1.0 / vm;
        pm0 = vmerge * pm0;
        pm1 = vmerge * pm1;
        pm0 = x0 + pm0;
        pm1 = y0 + pm1;
        pm2 = vmerge * pm2;
        pm0 = pm0 - P.extent[0] * (double)(int)((pm0 - P.center[0]) * P.hli[0]);
        pm1 = pm1 - P.extent[1] * (double)(int)((pm1 - P.center[1]) * P.hli[1]);
        bm = vmerge * bm;
        hm = vmerge * hm;
        for (int k = 0; k < 3; ++k) wm[k] = vmerge * wm[k];
        // shape (parcel_merge.f90:263-322)
        double b[5];
        for (int k = 0; k < 5; ++k) b[k] = pv.get(A_B11 + k, ic);
        double B33 = get_B33<FastOps>(b, vic, err);
        double dx = pdelta(xic - pm0, P.extent[0], P.extenti[0]);
        double dy = pdelta(yic - pm1, P.extent[1], P.extenti[1]);
        double dz = zic - pm2;
        double mu = vic * vmerge;
        double Bm[6];
        Bm[0] = mu * (5.0 * (dx * dx) + b[0]);
        Bm[1] = mu * (5.0 * dx * dy + b[1]);
        Bm[2] = mu * (5.0 * dx * dz + b[2]);
        Bm[3] = mu * (5.0 * (dy * dy) + b[3]);
        Bm[4] = mu * (5.0 * dy * dz + b[4]);
        Bm[5] = mu * (5.0 * (dz * dz) + B33);
        for (int q = s0; q < s1; ++q) {
            int is = ism[svals[q]];
            double px = pv.get(A_X, is), py = pv.get(A_Y, is), pz = pv.get(A_Z, is);
            double ex = pdelta(px - pm0, P.extent[0], P.extenti[0]);
            double ey = pdelta(py - pm1, P.extent[1], P.extenti[1]);
            double ez = pz - pm2;
            double bs[5];
            for (int k = 0; k < 5; ++k) bs[k] = pv.get(A_B11 + k, is);
            double vs = pv.get(A_VOL, is);
            double B33s = get_B33<FastOps>(bs, vs, err);
            double m2 = vmerge * vs;
            Bm[0] = Bm[0] + m2 * (5.0 * (ex * ex) + bs[0]);
            Bm[1] = Bm[1] + m2 * (5.0 * ex * ey + bs[1]);
            Bm[2] = Bm[2] + m2 * (5.0 * ex * ez + bs[2]);
            Bm[3] = Bm[3] + m2 * (5.0 * (ey * ey) + bs[3]);
            Bm[4] = Bm[4] + m2 * (5.0 * ey * ez + bs[4]);
            Bm[5] = Bm[5] + m2 * (5.0 * (ez * ez) + B33s);
        }
        double detB = Bm[0] * (Bm[3] * Bm[5] - Bm[4] * Bm[4]) - Bm[1] * (Bm[1] * Bm[5] - Bm[2] * Bm[4])
                    + Bm[2] * (Bm[1] * Bm[4] - Bm[2] * Bm[3]);
        double abc = get_abc(vm);
        double factor = pow(abc * abc / detB, 1.0 / 3.0);
        pv.set(A_VOL, ic, vm);
        pv.set(A_X, ic, pm0);
        pv.set(A_Y, ic, pm1);
        pv.set(A_Z, ic, pm2);
        pv.set(A_BUOY, ic, bm);
        pv.set(A_HUM, ic, hm);
        for (int k = 0; k < 3; ++k) pv.set(A_VX + k, ic, wm[k]);
        for (int k = 0; k < 5; ++k) pv.set(A_B11 + k, ic, Bm[k] * factor);
        if (L.label) {
            L.label[ic] = labm;
            L.dil[ic] = dilm;
        }
    }
}

// parcel_delete (parcel_container.f90:413-458): the i-th hole (ascending,
// below the new count) receives the i-th surviving parcel from the top.
__global__ void k_mark_deleted(const int* ism, int nm, char* del) { MLOOP(nm) del[ism[i]] = 1; }
__global__ void k_src_flags(const char* del, int newN, int N, int* f) {
    MLOOP(N - newN) f[i] = del[newN + i] ? 0 : 1;
}
__global__ void k_hole_flags(const int* ism, int nm, int newN, int* f) { MLOOP(nm) f[i] = ism[i] < newN; }
// the first nattr attributes of the nh sources into the holes
__global__ void k_move(PView pv, const int* holes, const int* srcs, int nh, int newN, int nattr) {
    MLOOP((long long)nh * nattr) {
        int h = (int)(i % nh);
        int a = (int)(i / nh);
        int dst = holes[h];
        int src = newN + srcs[nh - 1 - h];
        pv.set(a, dst, pv.get(a, src));
    }
}

__global__ void k_move_rank(int* rank, const int* holes, const int* srcs, int nh, int newN) {
    MLOOP(nh) rank[holes[i]] = rank[newN + srcs[nh - 1 - i]];
}

__global__ void k_move_labels(long long* label, double* dil, const int* holes, const int* srcs, int nh, int newN) {
    MLOOP(nh) {
        const int dst = holes[i], src = newN + srcs[nh - 1 - i];
        label[dst] = label[src];
        dil[dst] = dil[src];
    }
}

__global__ void k_periodic_m(Params P, PView pv, long long n) {
    MLOOP(n) {
        double x = pv.get(A_X, i), y = pv.get(A_Y, i);
        pv.set(A_X, i, x - P.extent[0] * (double)(int)((x - P.center[0]) * P.hli[0]));
        pv.set(A_Y, i, y - P.extent[1] * (double)(int)((y - P.center[1]) * P.hli[1]));
    }
}

// Buffers of parcel_delete for N parcels of which nm go: del (N bytes);
// hf, holes, sf, sidx, srcs (nm ints each); with container indices (ord:
// slot of each container index) also hole_f, src_f, iota, holes_r, srcs_r (N
// ints each); CUB temporary storage for a selection over N items; 2 counters.
struct DeleteBufs {
    char* del;
    int *hf, *holes, *sf, *sidx, *srcs;
    int *hole_f, *src_f, *iota, *holes_r, *srcs_r;
    const int* ord;
    void* ctmp;
    size_t cubb;
    int* dcount;
};

static int read_int(Ctx& c, const int* d);

// parcel_delete (parcel_container.f90:413-458) of the nm parcels in slots
// ism (ascending where the slots are the container indices, keep_order = 1:
// the holes are filled in that order; state_only: the attributes a parcel
// carries between steps, the rest being dead inside a step's merge): the
// i-th hole (below the new count)
// receives the i-th surviving parcel from the top; with container indices the same rule runs
// on the indices (the slots are compacted the same way, and each parcel keeps
// the index the reference's container gives it).  Leaves c.n to the caller.
static void delete_slots(Ctx& c, int N, const int* ism, int nm, const DeleteBufs& b, bool state_only) {
    cudaStream_t st = c.stream;
    const int newN = N - nm;
    const int* ord = b.ord;
    const bool ranked = c.rank != nullptr;
    char* del = b.del;
    CK(cudaMemsetAsync(del, 0, N, st));
    k_mark_deleted<<<mgrid(nm), MB, 0, st>>>(ism, nm, del);
    CKL();
    if (ranked) {
        k_del_rank_flags<<<mgrid(N), MB, 0, st>>>(ord, del, N, newN, b.hole_f, b.src_f);
        CKL();
        k_iota<<<mgrid(N), MB, 0, st>>>(b.iota, N);
        CKL();
        size_t bb = b.cubb;
        CK(cub::DeviceSelect::Flagged(b.ctmp, bb, b.iota, b.hole_f, b.holes_r, b.dcount, N, st));
        bb = b.cubb;
        CK(cub::DeviceSelect::Flagged(b.ctmp, bb, b.iota, b.src_f, b.srcs_r, b.dcount + 1, N, st));
        const int nhr = read_int(c, b.dcount);
        if (nhr > 0) {
            k_rerank<<<mgrid(nhr), MB, 0, st>>>(ord, b.holes_r, b.srcs_r, nhr, c.rank);
            CKL();
        }
    }
    k_hole_flags<<<mgrid(nm), MB, 0, st>>>(ism, nm, newN, b.hf);
    CKL();
    {
        size_t bb = b.cubb;
        CK(cub::DeviceSelect::Flagged(b.ctmp, bb, ism, b.hf, b.holes, b.dcount, nm, st));
    }
    const int nh = read_int(c, b.dcount);
    if (nh > 0) {
        k_src_flags<<<mgrid(nm), MB, 0, st>>>(del, newN, N, b.sf);
        CKL();
        k_iota<<<mgrid(nm), MB, 0, st>>>(b.sidx, nm);
        CKL();
        size_t bb = b.cubb;
        CK(cub::DeviceSelect::Flagged(b.ctmp, bb, b.sidx, b.sf, b.srcs, b.dcount + 1, N - newN, st));
        const int nattr = state_only ? N_STATE : N_ATTR;
        k_move<<<mgrid((long long)nh * nattr), MB, 0, st>>>(c.pv, b.holes, b.srcs, nh, newN, nattr);
        CKL();
        if (ranked) {
            k_move_rank<<<mgrid(nh), MB, 0, st>>>(c.rank, b.holes, b.srcs, nh, newN);
            CKL();
        }
        if (c.label) {
            k_move_labels<<<mgrid(nh), MB, 0, st>>>(c.label, c.dil, b.holes, b.srcs, nh, newN);
            CKL();
        }
    }
}

// ---------------------------------------------------------------------------
struct Arena {
    char* base;
    size_t off, cap;
    template <class T>
    T* take(size_t n) {
        off = (off + 255) & ~(size_t)255;
        T* p = reinterpret_cast<T*>(base + off);
        off += sizeof(T) * std::max<size_t>(n, 1);
        if (off > cap) throw CudaError(EPIC_ERR_CAPACITY, "merge scratch arena overflow");
        return p;
    }
};

static int read_int(Ctx& c, const int* d) {
    int h = 0;
    CK(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return h;
}

static size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

// Scratch bytes of the merge's binning phase for n parcels.
size_t merge_scratch_bytes(long long n) {
    size_t cub1 = 0;
    cub::DeviceSelect::Flagged(nullptr, cub1, (int*)0, (int*)0, (int*)0, (int*)0, (int)n);
    return al(sizeof(int) * (size_t)n) * 7 + al(cub1) + 4096;
}

long long parcel_merge(Ctx& c, bool in_step) {
    const Params& P = c.P;
    const int N = (int)c.n;
    c.n_pairs = 0;
    if (N == 0) return 0;
    Box B;
    B.hs1 = P.nx + 3;
    B.hs2 = P.ny + 3;
    B.hncell = (long long)B.hs1 * B.hs2 * (P.nz + 2);
    cudaStream_t st = c.stream;
    unsigned* err = &c.dsc->err;

    // ---- phase 1: binning and the local small list (parcel_nearest.f90:416-431)
    prof_begin(c, "merge_bin");
    size_t cub1 = 0;
    cub::DeviceSelect::Flagged(nullptr, cub1, (int*)0, (int*)0, (int*)0, (int*)0, N, st);
    size_t bytes1 = merge_scratch_bytes(N);
    Arena a1{reinterpret_cast<char*>(c.get_scratch2(bytes1)), 0, bytes1};
    int* cell0 = a1.take<int>(N);
    int* small = a1.take<int>(N);
    unsigned* bits = a1.take<unsigned>(N);
    int* Ls = a1.take<int>(N);
    int* idx = a1.take<int>(N);
    int* dcount = a1.take<int>(8);
    void* tmp1 = a1.take<char>(cub1);
    // box-ordered store: the small parcels (merge index m), the cell lists and
    // parcel_delete follow the container indices in c.rank
    const bool ranked = c.rank != nullptr;
    int* ord = ranked ? a1.take<int>(N) : nullptr;
    int* smallr = ranked ? a1.take<int>(N) : nullptr;
    k_bin_locals<<<mgrid(N), MB, 0, st>>>(P, B, c.pv, N, cell0, small, bits, err);
    CKL();
    if (ranked) {
        container_order(c, ord);
        k_by_rank<<<mgrid(N), MB, 0, st>>>(ord, small, N, smallr);
        CKL();
        CK(cub::DeviceSelect::Flagged(tmp1, cub1, ord, smallr, Ls, dcount, N, st));
    } else {
        k_iota<<<mgrid(N), MB, 0, st>>>(idx, N);
        CKL();
        CK(cub::DeviceSelect::Flagged(tmp1, cub1, idx, small, Ls, dcount, N, st));
    }
    const int nls = read_int(c, dcount);
    prof_end(c, "merge_bin");
    if (nls == 0) {
        k_periodic_m<<<mgrid(N), MB, 0, st>>>(P, c.pv, N);
        CKL();
        return 0;
    }

    // ---- phase 2: copies, sort, search, tree, merge, delete
    const long long ncp_max = 3LL * nls;
    const long long NTm = (long long)N + ncp_max;
    size_t c_sort = 0, c_scan = 0, c_sel = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, c_sort, (int*)0, (int*)0, (int*)0, (int*)0, (int)NTm, 0, 32, st);
    cub::DeviceScan::ExclusiveSum(nullptr, c_scan, (int*)0, (int*)0, (int)(8LL * nls + 1), st);
    cub::DeviceSelect::Flagged(nullptr, c_sel, (int*)0, (int*)0, (int*)0, (int*)0, nls, st);
    size_t c_sel_n = 0;
    if (ranked) cub::DeviceSelect::Flagged(nullptr, c_sel_n, (int*)0, (int*)0, (int*)0, (int*)0, N, st);
    size_t cubb = std::max({c_sort, c_scan, c_sel, c_sel_n});
    size_t bytes2 = al(sizeof(int) * NTm) * 4                       // cell, vals, skeys, svals
                  + al(sizeof(int) * (8 * (size_t)nls + 1)) * 3       // F, off, copyidx
                  + al(sizeof(double) * ncp_max) * 3 + al(sizeof(int) * ncp_max) * 2   // copies
                  + al(sizeof(int) * B.hncell) * 2                    // cell ranges
                  + al(sizeof(int) * (size_t)nls) * 14 + al(sizeof(double) * (size_t)nls)
                  + al(sizeof(int) * ((size_t)nls + ncp_max)) * 4       // search order
                  + al((size_t)N) * 3 + al(sizeof(int) * (size_t)N)    // tree flags, minv
                  + al(cubb) + 64 * 256;
    Arena ar{reinterpret_cast<char*>(c.get_scratch(bytes2)), 0, bytes2};
    void* ctmp = ar.take<char>(cubb);
    int* cell = ar.take<int>(NTm);
    int* vals = ar.take<int>(NTm);
    int* skeys = ar.take<int>(NTm);
    int* svals = ar.take<int>(NTm);
    int* F = ar.take<int>(8 * (size_t)nls + 1);
    int* off = ar.take<int>(8 * (size_t)nls + 1);
    int* copyidx = ar.take<int>(8 * (size_t)nls);
    CopyArgs C;
    C.cx = ar.take<double>(ncp_max);
    C.cy = ar.take<double>(ncp_max);
    C.cz = ar.take<double>(ncp_max);
    C.pid = ar.take<int>(ncp_max);
    C.mid = ar.take<int>(ncp_max);
    int* cstart = ar.take<int>(B.hncell);
    int* cend = ar.take<int>(B.hncell);

    prof_begin(c, "merge_cells");
    if (ranked) {
        k_rank_cells<<<mgrid(N), MB, 0, st>>>(ord, cell0, N, cell, vals);
        CKL();
    } else {
        CK(cudaMemcpyAsync(cell, cell0, sizeof(int) * (size_t)N, cudaMemcpyDeviceToDevice, st));
    }
    k_copy_flags<<<mgrid(8LL * nls), MB, 0, st>>>(Ls, nls, bits, F);
    CKL();
    CK(cudaMemsetAsync(F + 8LL * nls, 0, sizeof(int), st));
    {
        size_t b = cubb;
        CK(cub::DeviceScan::ExclusiveSum(ctmp, b, F, off, 8 * nls + 1, st));
    }
    const int ncp = read_int(c, off + 8LL * nls);
    const long long NT = (long long)N + ncp;
    CK(cudaMemsetAsync(copyidx, 0xff, sizeof(int) * 8 * (size_t)nls, st));
    k_make_copies<<<mgrid(8LL * nls), MB, 0, st>>>(P, B, c.pv, Ls, nls, F, off, C, cell + N, copyidx, err);
    CKL();
    // locals in container order (their slots), then the copies N + q
    if (ranked) k_iota_from<<<mgrid(ncp), MB, 0, st>>>(vals + N, ncp, N);
    else k_iota<<<mgrid(NT), MB, 0, st>>>(vals, NT);
    CKL();
    int endbit = 1;
    while ((1LL << endbit) < B.hncell) ++endbit;
    {
        size_t b = cubb;
        CK(cub::DeviceRadixSort::SortPairs(ctmp, b, cell, skeys, vals, svals, (int)NT, 0, endbit, st));
    }
    CK(cudaMemsetAsync(cstart, 0, sizeof(int) * B.hncell, st));
    CK(cudaMemsetAsync(cend, 0, sizeof(int) * B.hncell, st));
    k_cell_ranges<<<mgrid(NT), MB, 0, st>>>(skeys, NT, cstart, cend);
    CKL();
    prof_end(c, "merge_cells");
    prof_begin(c, "merge_search");

    int* iclo = ar.take<int>((size_t)nls + ncp);
    double* dclo = ar.take<double>((size_t)nls + ncp);
    // the second parcel store (free between the step's sorts) holds the
    // sorted entries' positions when there is one
    double4* sp = nullptr;
    if (c.pv_alt && (size_t)NT * sizeof(double4) <= c.store_bytes()) {
        sp = reinterpret_cast<double4*>(c.pv_alt);
        k_sorted_pos<<<mgrid(NT), MB, 0, st>>>(c.pv, C, N, svals, NT, sp);
        CKL();
    }
    // the small entries in cell order
    const int nse = nls + ncp;
    int* okeys = ar.take<int>(nse);
    int* ovals = ar.take<int>(nse);
    int* skeys2 = ar.take<int>(nse);
    int* order = ar.take<int>(nse);
    k_small_keys<<<mgrid(nse), MB, 0, st>>>(Ls, nls, ncp, cell0, cell + N, okeys, ovals);
    CKL();
    {
        size_t b = cubb;
        CK(cub::DeviceRadixSort::SortPairs(ctmp, b, okeys, skeys2, ovals, order, nse, 0, endbit, st));
    }
    k_search<<<mgrid((long long)nse), MB, 0, st>>>(P, B, c.pv, C, N, Ls, nls, ncp, svals, sp, order, cstart,
                                                   cend, iclo, dclo);
    CKL();
    k_globally<<<mgrid(nls), MB, 0, st>>>(nls, copyidx, iclo, dclo, err);
    CKL();
    check_device_error(c);
    prof_end(c, "merge_search");

    // resolve_tree
    char* merged = ar.take<char>(N);
    char* leaf = ar.take<char>(N);
    char* avail = ar.take<char>(N);
    CK(cudaMemsetAsync(merged, 0, N, st));
    CK(cudaMemsetAsync(leaf, 0, N, st));
    CK(cudaMemsetAsync(avail, 0, N, st));
    const int g = mgrid(nls);
    for (int it = 0;; ++it) {
        prof_begin(c, "merge_tree1");
        CK(cudaMemsetAsync(dcount, 0, sizeof(int), st));
        k_tree_a<<<g, MB, 0, st>>>(Ls, iclo, nls, merged, leaf, avail);
        CKL();
        k_tree_b<<<g, MB, 0, st>>>(Ls, iclo, nls, merged, leaf);
        CKL();
        k_tree_c<<<g, MB, 0, st>>>(Ls, iclo, nls, merged, leaf, avail);
        CKL();
        k_tree_d<<<g, MB, 0, st>>>(Ls, iclo, nls, merged, leaf, avail, dcount);
        CKL();
        const int more = read_int(c, dcount);
        prof_end(c, "merge_tree1");
        if (!more) break;
        if (it > 1000000) throw CudaError(EPIC_ERR_TIMEOUT, "resolve_tree: stage 1 did not terminate");
    }
    char* dom = ar.take<char>(nls);
    char* status = ar.take<char>(nls);
    int* minv = ar.take<int>(N);
    CK(cudaMemsetAsync(minv, 0xff, sizeof(int) * (size_t)N, st));
    k_set_minv<<<g, MB, 0, st>>>(Ls, nls, minv);
    CKL();
    k_tree_e<<<g, MB, 0, st>>>(Ls, iclo, nls, merged, leaf, avail);
    CKL();
    k_tree_f_init<<<g, MB, 0, st>>>(Ls, iclo, nls, merged, leaf, avail, dom, status, err);
    CKL();
    for (int it = 0;; ++it) {
        prof_begin(c, "merge_tree2");
        CK(cudaMemsetAsync(dcount, 0, sizeof(int), st));
        k_tree_f_round<<<g, MB, 0, st>>>(iclo, nls, minv, avail, status, dcount);
        CKL();
        const int more = read_int(c, dcount);
        prof_end(c, "merge_tree2");
        if (!more) break;
        if (it > 1000000) throw CudaError(EPIC_ERR_TIMEOUT, "resolve_tree: stage 2 did not terminate");
    }
    k_tree_f_apply<<<g, MB, 0, st>>>(Ls, nls, status, avail, dom);
    CKL();
    k_tree_g<<<g, MB, 0, st>>>(iclo, nls, status, avail, dom);
    CKL();
    check_device_error(c);

    // merging pairs in m order
    prof_begin(c, "merge_group");
    int* domi = ar.take<int>((size_t)nls + 1);
    int* dpos = ar.take<int>((size_t)nls + 1);
    k_char_to_int<<<g, MB, 0, st>>>(dom, domi, nls);
    CKL();
    CK(cudaMemsetAsync(domi + nls, 0, sizeof(int), st));
    {
        size_t b = cubb;
        CK(cub::DeviceScan::ExclusiveSum(ctmp, b, domi, dpos, nls + 1, st));
    }
    const int nm = read_int(c, dpos + nls);
    if (nm == 0) {
        prof_end(c, "merge_group");
        k_periodic_m<<<mgrid(N), MB, 0, st>>>(P, c.pv, N);
        CKL();
        return 0;
    }
    const long long call = c.merge_calls++;
    int* ism = ar.take<int>(nm);
    int* icl = ar.take<int>(nm);
    k_pack_pairs<<<g, MB, 0, st>>>(Ls, iclo, nls, dom, dpos, ism, icl);
    CKL();
    {
        // the pairs as container indices
        const int* pi = ism;
        const int* pc = icl;
        if (ranked) {
            int* ri = ar.take<int>(nm);
            int* rc = ar.take<int>(nm);
            k_pairs_rank<<<mgrid(nm), MB, 0, st>>>(c.rank, ism, icl, nm, ri, rc);
            CKL();
            pi = ri;
            pc = rc;
        }
        if (2LL * nm > c.pairs_cap) {
            if (c.pairs_dev) CK(cudaFreeAsync(c.pairs_dev, st));
            c.pairs_dev = nullptr;
            c.pairs_cap = 0;
            const long long cap = 3LL * nm + 1024;
            CK(cudaMallocAsync(&c.pairs_dev, sizeof(int) * (size_t)cap, st));
            c.pairs_cap = cap;
        }
        CK(cudaMemcpyAsync(c.pairs_dev, pi, sizeof(int) * nm, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(c.pairs_dev + nm, pc, sizeof(int) * nm, cudaMemcpyDeviceToDevice, st));
        c.n_pairs = nm;
    }

    // collect_merge_stats (parcel_merge.f90:365-394)
    unsigned long long* bigc = ar.take<unsigned long long>(1);
    CK(cudaMemsetAsync(bigc, 0, sizeof(unsigned long long), st));
    k_big_close<<<mgrid(nm), MB, 0, st>>>(c.pv, icl, nm, P.vmin, bigc);
    CKL();

    // groups by ic; the stable sort keeps m order inside a group
    int* mvals = ar.take<int>(nm);
    int* gk = ar.take<int>(nm);
    int* gv = ar.take<int>(nm);
    int* head = ar.take<int>(nm);
    int* gidx = ar.take<int>(nm);
    int* gstart = ar.take<int>(nm);
    k_iota<<<mgrid(nm), MB, 0, st>>>(mvals, nm);
    CKL();
    int nbits = 1;
    while ((1LL << nbits) <= N) ++nbits;
    {
        size_t b = cubb;
        CK(cub::DeviceRadixSort::SortPairs(ctmp, b, icl, gk, mvals, gv, nm, 0, nbits, st));
    }
    k_group_heads<<<mgrid(nm), MB, 0, st>>>(gk, nm, head);
    CKL();
    k_iota<<<mgrid(nm), MB, 0, st>>>(gidx, nm);
    CKL();
    {
        size_t b = cubb;
        CK(cub::DeviceSelect::Flagged(ctmp, b, gidx, head, gstart, dcount, nm, st));
    }
    const int ng = read_int(c, dcount);
    const MergeLabels ML{c.label, c.dil, c.cfg.label_seed, call};
    k_group_merge<<<mgrid(ng), MB, 0, st>>>(P, c.pv, gstart, ng, nm, gk, gv, ism, ML, err);
    CKL();

    prof_end(c, "merge_group");
    // parcel_delete
    prof_begin(c, "merge_delete");
    const int newN = N - nm;
    {
        DeleteBufs db;
        db.del = merged;
        db.hf = head; db.holes = gidx; db.sf = mvals; db.sidx = gk; db.srcs = gv;
        // with container indices: the binning arrays are free now (the group
        // merge reads gk, gv and ism)
        db.hole_f = cell; db.src_f = vals; db.iota = skeys; db.holes_r = svals; db.srcs_r = svals + N;
        db.ord = ord; db.ctmp = ctmp; db.cubb = cubb; db.dcount = dcount;
        delete_slots(c, N, ism, nm, db, in_step);
    }
    unsigned long long hb = 0;
    CK(cudaMemcpyAsync(&hb, bigc, sizeof(hb), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    c.n_big_close += (long long)hb;
    c.n = newN;
    c.n_box = std::min<long long>(c.n_box, newN);   // holes below newN now hold parcels from the end
    c.n_parcel_merges += nm;
    k_periodic_m<<<mgrid(newN), MB, 0, st>>>(P, c.pv, newN);
    CKL();
    prof_end(c, "merge_delete");
    return nm;
}

__global__ void k_slots_of(const int* ord, const int* idx, int n, int* ism) {
    MLOOP(n) ism[i] = ord ? ord[idx[i]] : idx[i];
}

// parcel_delete alone (test hook): idx holds nm distinct container indices
// (0-based), host memory.
void test_delete(Ctx& c, const int* idx, int nm) {
    const int N = (int)c.n;
    if (nm <= 0) return;
    if (nm > N) throw CudaError(EPIC_ERR_ARG, "delete: more parcels than there are");
    size_t cubb = 0;
    cub::DeviceSelect::Flagged(nullptr, cubb, (int*)0, (int*)0, (int*)0, (int*)0, N, c.stream);
    std::vector<void*> mem;
    auto grab = [&](size_t bytes) {
        void* p = nullptr;
        CK(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
        mem.push_back(p);
        return p;
    };
    try {
        DeleteBufs b;
        int* didx = static_cast<int*>(grab(sizeof(int) * nm));
        int* ism = static_cast<int*>(grab(sizeof(int) * nm));
        b.del = static_cast<char*>(grab(N));
        b.hf = static_cast<int*>(grab(sizeof(int) * nm));
        b.holes = static_cast<int*>(grab(sizeof(int) * nm));
        b.sf = static_cast<int*>(grab(sizeof(int) * nm));
        b.sidx = static_cast<int*>(grab(sizeof(int) * nm));
        b.srcs = static_cast<int*>(grab(sizeof(int) * nm));
        int* ord = nullptr;
        b.hole_f = b.src_f = b.iota = b.holes_r = b.srcs_r = nullptr;
        if (c.rank) {
            ord = static_cast<int*>(grab(sizeof(int) * N));
            b.hole_f = static_cast<int*>(grab(sizeof(int) * N));
            b.src_f = static_cast<int*>(grab(sizeof(int) * N));
            b.iota = static_cast<int*>(grab(sizeof(int) * N));
            b.holes_r = static_cast<int*>(grab(sizeof(int) * N));
            b.srcs_r = static_cast<int*>(grab(sizeof(int) * N));
            container_order(c, ord);
        }
        b.ord = ord;
        b.ctmp = grab(cubb);
        b.cubb = cubb;
        b.dcount = static_cast<int*>(grab(sizeof(int) * 2));
        // ascending, as parcel_delete takes them
        std::vector<int> sorted(idx, idx + nm);
        std::sort(sorted.begin(), sorted.end());
        CK(cudaMemcpyAsync(didx, sorted.data(), sizeof(int) * nm, cudaMemcpyHostToDevice, c.stream));
        k_slots_of<<<mgrid(nm), MB, 0, c.stream>>>(ord, didx, nm, ism);
        CKL();
        delete_slots(c, N, ism, nm, b, false);
        CK(cudaStreamSynchronize(c.stream));   // before the host copy of the indices goes
        c.n = N - nm;
        c.n_box = std::min<long long>(c.n_box, c.n);
    } catch (...) {
        cudaStreamSynchronize(c.stream);
        for (void* p : mem) cudaFree(p);
        throw;
    }
    for (void* p : mem) cudaFree(p);
}

}  // namespace epic
