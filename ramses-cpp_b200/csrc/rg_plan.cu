// rg_plan.cu -- integer work of the level step, built once per topology.
//
// Reference behaviour reproduced bit-exactly (paths relative to RAMSES-CPP):
//   level list order         HydroSolver.cpp:43-47 (walk of headl/next)
//   cell_levels              HydroSolver.cpp:22-38
//   get_nbor_grids/cells     AmrGrid.cpp:389-444 (iii/jjj of Constants.cpp:8-43)
//   get_nbor_cells_coarse    AmrGrid.cpp:513-550 (periodic; nboundary == 0)
//   interface branches       HydroSolver.cpp:118-162, reflux test :476
//   CPU update order         HydroSolver.cpp:565-572 (octs, ic, idim, side)
#include <algorithm>
#include <climits>
#include <cstdio>

#include "rg_internal.cuh"
#include "rg_nav.cuh"

namespace rg {

namespace {

constexpr int TPB = 256;
inline int nblk(long long n, int tpb = TPB) { return (int)std::max(1LL, std::min((n + tpb - 1) / tpb, 1LL << 30)); }

// Neighbour of an arbitrary cell id, as the ghost branch looks it up
// (HydroSolver.cpp:179-187).
__device__ __forceinline__ int nbor_of_cell(const TreeView& T, int id, int idim, int side, DevStatus* st) {
    if (id <= T.ncoarse) return coarse_nbor(T, id, idim, side);
    int ig = ((id - T.ncoarse - 1) % T.ngridmax) + 1;
    int ic = ((id - T.ncoarse - 1) / T.ngridmax) + 1;
    return nbor_cell_dir(T, ig, ic, idim, side, st);
}

// ---------------------------------------------------------------- list ranking
__global__ void k_rank_init(const int* __restrict__ next, int n, int* jump, int* dist) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int nx = next[i];
        bool ok = nx >= 1 && nx <= n;
        jump[i] = ok ? nx - 1 : i;
        dist[i] = ok ? 1 : 0;
    }
}
__global__ void k_rank_step(int n, const int* __restrict__ j0, const int* __restrict__ d0, int* j1, int* d1) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int j = j0[i];
        j1[i] = j0[j];
        d1[i] = d0[i] + d0[j];
    }
}
__global__ void k_rank_check(int n, const int* __restrict__ jump, const int* __restrict__ dist, DevStatus* st) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int j = jump[i];
        if (jump[j] != j || dist[j] != 0) raise_err(st, DE_TOPO_CYCLE, i + 1);
    }
}

__global__ void k_cell_levels(TreeView T, int* cell_level, int ttd, DevStatus* st) {
    for (int ig = blockIdx.x * blockDim.x + threadIdx.x + 1; ig <= T.ngridmax; ig += gridDim.x * blockDim.x) {
        if (T.father[ig - 1] <= 0) continue;
        int level = 1, curr = ig, guard = 0;
        while (curr > 0) {
            int fc = T.father[curr - 1];
            if (fc <= T.ncoarse) break;
            curr = ((fc - T.ncoarse - 1) % T.ngridmax) + 1;
            level++;
            if (++guard > 4096) {
                raise_err(st, DE_TOPO_CYCLE, ig);
                break;
            }
        }
        for (int ic = 1; ic <= ttd; ++ic) cell_level[T.ncoarse + (ic - 1) * T.ngridmax + ig] = level;
    }
}

// count[0]: octs found; check_on_device: the block that finishes last
// (count[1] counts finished blocks) compares count[0] with noct itself -- a
// shorter chain than the level count says raises DE_LIST -- so the host
// need not read it back
__global__ void k_level_octs(int n, const int* __restrict__ jump, const int* __restrict__ dist, int head0, int noct,
                             int* octs, int* count, DevStatus* st, bool check_on_device) {
    int tail = jump[head0];
    int dh = dist[head0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (jump[i] != tail) continue;
        int pos = dh - dist[i];
        if (pos < 0 || pos >= noct) {
            raise_err(st, DE_LIST, i + 1);
            continue;
        }
        octs[pos] = i + 1;
        atomicAdd(count, 1);
    }
    if (!check_on_device) return;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(count + 1, 1) == (int)gridDim.x - 1 && atomicAdd(count, 0) != noct) raise_err(st, DE_LIST, noct);
    }
}

// ---------------------------------------------------------------- plan cells
__device__ __forceinline__ int plan_cell_id(const TreeView& T, const int* octs, int level0, int noct, int p) {
    if (level0) return p + 1;
    int icx = p / noct, k = p - icx * noct;
    return T.ncoarse + icx * T.ngridmax + octs[k];
}

__global__ void k_plan_cpos(TreeView T, const int* __restrict__ octs, int level0, int noct, int ncells, int* cpos) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < ncells; p += gridDim.x * blockDim.x)
        cpos[plan_cell_id(T, octs, level0, noct, p)] = p;
}

template <int NDIM>
__global__ void k_plan_cells(TreeView T, const int* __restrict__ octs, int level0, int ilevel, int noct, int ncells,
                             const int* __restrict__ cpos, int* icn, int* stc, int8_t* kind,
                             unsigned long long* nactive, DevStatus* st) {
    constexpr int NS = 2 * NDIM;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < ncells; p += gridDim.x * blockDim.x) {
        int c = plan_cell_id(T, octs, level0, noct, p);
        int icx = level0 ? 0 : p / noct;
        int ig = level0 ? 0 : octs[p - icx * noct];
        bool active = T.son[c - 1] == 0;
        if (active) atomicAdd(nactive, 1ULL);
        for (int s = 0; s < NS; ++s) {
            int idim = s >> 1, side = s & 1;
            int n = level0 ? coarse_nbor(T, c, idim, side) : nbor_cell_dir(T, ig, icx + 1, idim, side, st);
            icn[(size_t)s * ncells + p] = n;
            int kd = K_NONE, nl = 0, nr = 0;
            if (active) {
                if (n > T.ncell) {
                    raise_err(st, DE_BAD_INDEX, c);
                    n = 0;
                }
                int nlev = (n > 0) ? T.cell_level[n] : 0;
                if (n > 0 && (T.son[n - 1] > 0 || nlev > ilevel)) {
                    kd = K_ZERO;
                } else if (n <= 0) {
                    int ib = -n;
                    int btype = 1;
                    if (ib > 0 && ib <= T.nbound_type && T.bound_type) btype = T.bound_type[ib - 1];
                    kd = K_BOUND | (btype == 1 ? KIND_REFLECT : 0);
                } else if (nlev == ilevel) {  // son[n-1] == 0 here
                    if (cpos[n] < 0) raise_err(st, DE_SAME_OUTSIDE, n);
                    kd = K_SAME;
                } else {
                    kd = K_GHOST;
                }
                if ((kd & KIND_MASK) == K_SAME || (kd & KIND_MASK) == K_GHOST) {
                    if (!level0) {
                        nl = nbor_of_cell(T, n, idim, 0, st);
                        nr = nbor_of_cell(T, n, idim, 1, st);
                    }
                    if (nlev < ilevel) kd |= KIND_REFLUX;
                }
            }
            kind[(size_t)s * ncells + p] = (int8_t)kd;
            stc[((size_t)s * 2 + 0) * ncells + p] = nl;
            stc[((size_t)s * 2 + 1) * ncells + p] = nr;
        }
    }
}

// Cells outside the level whose primitives the step reads.
template <int NDIM>
__global__ void k_plan_xprim(int ncells, const int* __restrict__ cpos, const int* __restrict__ icn,
                             const int* __restrict__ stc, const int8_t* __restrict__ kind, int* pmark, int* xprim,
                             int* nx) {
    constexpr int NS = 2 * NDIM;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < ncells; p += gridDim.x * blockDim.x) {
        if (kind[p] == K_NONE) continue;  // inactive cell (slot 0 is NONE iff inactive)
        for (int s = 0; s < NS; ++s) {
            int refs[3] = {icn[(size_t)s * ncells + p], stc[((size_t)s * 2) * ncells + p],
                           stc[((size_t)s * 2 + 1) * ncells + p]};
            for (int r = 0; r < 3; ++r) {
                int id = refs[r];
                if (id <= 0 || cpos[id] >= 0) continue;
                if (atomicCAS(&pmark[id], 0, 1) == 0) xprim[atomicAdd(nx, 1)] = id;
            }
        }
    }
}

// ---------------------------------------------------------------- events
__device__ __forceinline__ int cpu_key(int level0, int ttd, int noct, int p, int slot) {
    if (level0) return p * 8 + slot;
    int icx = p / noct, k = p - icx * noct;
    return (k * ttd + icx) * 8 + slot;
}

template <int NDIM>
__global__ void k_ev_claim(int ncells, const int* __restrict__ cpos, const int* __restrict__ icn,
                           const int8_t* __restrict__ kind, int* tmap, int* textra, int* nextra) {
    constexpr int NS = 2 * NDIM;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < ncells; p += gridDim.x * blockDim.x) {
        for (int s = 0; s < NS; ++s) {
            if (!(kind[(size_t)s * ncells + p] & KIND_REFLUX)) continue;
            int n = icn[(size_t)s * ncells + p];
            if (cpos[n] >= 0) continue;
            if (atomicCAS(&tmap[n], -1, -2) == -1) {
                int j = atomicAdd(nextra, 1);
                textra[j] = n;
                tmap[n] = ncells + j;
            }
        }
    }
}

__device__ __forceinline__ int target_of(const int* cpos, const int* tmap, int n) {
    int t = cpos[n];
    return t >= 0 ? t : tmap[n];
}

template <int NDIM>
__global__ void k_ev_count(int ncells, const int* __restrict__ cpos, const int* __restrict__ tmap,
                           const int* __restrict__ icn, const int8_t* __restrict__ kind, int* cnt) {
    constexpr int NS = 2 * NDIM;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < ncells; p += gridDim.x * blockDim.x) {
        if (kind[p] == K_NONE) continue;
        atomicAdd(&cnt[p], 1);  // own update
        for (int s = 0; s < NS; ++s) {
            if (!(kind[(size_t)s * ncells + p] & KIND_REFLUX)) continue;
            atomicAdd(&cnt[target_of(cpos, tmap, icn[(size_t)s * ncells + p])], 1);
        }
    }
}

template <int NDIM>
__global__ void k_ev_fill(int ncells, int level0, int noct, const int* __restrict__ cpos, const int* __restrict__ tmap,
                          const int* __restrict__ icn, const int8_t* __restrict__ kind, const int* __restrict__ off,
                          int* fillc, int* ev) {
    constexpr int NS = 2 * NDIM, TTD = 1 << NDIM;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < ncells; p += gridDim.x * blockDim.x) {
        if (kind[p] == K_NONE) continue;
        ev[off[p] + atomicAdd(&fillc[p], 1)] = cpu_key(level0, TTD, noct, p, OWN_SLOT);
        for (int s = 0; s < NS; ++s) {
            if (!(kind[(size_t)s * ncells + p] & KIND_REFLUX)) continue;
            int t = target_of(cpos, tmap, icn[(size_t)s * ncells + p]);
            ev[off[t] + atomicAdd(&fillc[t], 1)] = cpu_key(level0, TTD, noct, p, s);
        }
    }
}

// targets whose event count exceeds `limit`, appended to out (count in *n);
// the targets are the level's nc cells and the *nextra extra ones
__global__ void k_long_targets(int nc, const int* __restrict__ nextra, const int* __restrict__ off, int limit, int* out,
                               int* n) {
    const int ntarg = nc + *nextra;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntarg; t += gridDim.x * blockDim.x)
        if (off[t + 1] - off[t] > limit) out[atomicAdd(n, 1)] = t;
}

// each target's events into ascending key order (the CPU order), one thread
// per target; targets with more than `skip_above` events are left to
// k_ev_sort_long
__global__ void k_ev_sort(int nc, const int* __restrict__ nextra, const int* __restrict__ off, int* ev,
                          int skip_above) {
    const int ntarg = nc + *nextra;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntarg; t += gridDim.x * blockDim.x) {
        int a = off[t], b = off[t + 1];
        if (b - a > skip_above) continue;
        for (int i = a + 1; i < b; ++i) {
            int v = ev[i], j = i - 1;
            while (j >= a && ev[j] > v) {
                ev[j + 1] = ev[j];
                --j;
            }
            ev[j + 1] = v;
        }
    }
}

// The long targets' events (list and count from k_long_targets), one block
// per target: a bitonic network in shared memory.  Keys are distinct (one per
// source cell and slot), so any correct sort gives k_ev_sort's order; a
// target with more than kSortMax events falls back to one thread's
// insertion sort.
constexpr int kSortMax = 2048, kSortThreads = 256;
__global__ void __launch_bounds__(kSortThreads)
    k_ev_sort_long(const int* __restrict__ tlong, const int* __restrict__ nlong, const int* __restrict__ off, int* ev) {
    __shared__ int sh[kSortMax];
    const int n_long = *nlong;
    for (int w = blockIdx.x; w < n_long; w += gridDim.x) {
        const int t = tlong[w], a = off[t], n = off[t + 1] - a;
        if (n > kSortMax) {
            if (threadIdx.x == 0)
                for (int i = a + 1; i < a + n; ++i) {
                    const int v = ev[i];
                    int j = i - 1;
                    for (; j >= a && ev[j] > v; --j) ev[j + 1] = ev[j];
                    ev[j + 1] = v;
                }
            __syncthreads();
            continue;
        }
        int m = 1;
        while (m < n) m <<= 1;
        for (int i = threadIdx.x; i < m; i += blockDim.x) sh[i] = i < n ? ev[a + i] : INT_MAX;
        __syncthreads();
        for (int k = 2; k <= m; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < m; i += blockDim.x) {
                    const int ixj = i ^ j;
                    if (ixj > i) {
                        const int x = sh[i], y = sh[ixj];
                        if ((x > y) == ((i & k) == 0)) {
                            sh[i] = y;
                            sh[ixj] = x;
                        }
                    }
                }
                __syncthreads();
            }
        for (int i = threadIdx.x; i < n; i += blockDim.x) ev[a + i] = sh[i];
        __syncthreads();
    }
}

// ---------------------------------------------------------------- exclusive scan
constexpr int SCAN_TPB = 512;
constexpr int SCAN_ITEMS = SCAN_TPB * 2;

__device__ __forceinline__ int block_scan_excl(int v, int* sh, int* total) {
    int tid = threadIdx.x;
    sh[tid] = v;
    __syncthreads();
    for (int off = 1; off < blockDim.x; off <<= 1) {
        int t = (tid >= off) ? sh[tid - off] : 0;
        __syncthreads();
        sh[tid] += t;
        __syncthreads();
    }
    int incl = sh[tid];
    if (total) *total = sh[blockDim.x - 1];
    __syncthreads();
    return incl - v;
}

// Each block scans SCAN_ITEMS entries (2 per thread) and writes its total.
__global__ void k_scan_blocks(const int* __restrict__ in, int* out, int n, int* sums) {
    __shared__ int sh[SCAN_TPB];
    long long base = (long long)blockIdx.x * SCAN_ITEMS;
    long long i0 = base + 2 * threadIdx.x;
    int a = (i0 < n) ? in[i0] : 0, b = (i0 + 1 < n) ? in[i0 + 1] : 0;
    int tot;
    int e = block_scan_excl(a + b, sh, &tot);
    if (i0 < n) out[i0] = e;
    if (i0 + 1 < n) out[i0 + 1] = e + a;
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}
// Single block: exclusive scan of the block totals, sequential over chunks.
__global__ void k_scan_sums(int* sums, int nb, int* grand) {
    __shared__ int sh[SCAN_TPB];
    int carry = 0;
    for (int base = 0; base < nb; base += SCAN_TPB) {
        int i = base + threadIdx.x;
        int v = (i < nb) ? sums[i] : 0;
        int tot;
        int e = block_scan_excl(v, sh, &tot);
        if (i < nb) sums[i] = e + carry;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *grand = carry;
}
__global__ void k_scan_add(int* out, int n, const int* __restrict__ sums) {
    long long i = (long long)blockIdx.x * SCAN_ITEMS + threadIdx.x;
    int add = sums[blockIdx.x];
    if (i < n) out[i] += add;
    if (i + SCAN_TPB < n) out[i + SCAN_TPB] += add;
}

template <int NDIM>
int build_plan_t(rg_ctx* c, int ilevel, Plan& P);

}  // namespace

TreeView tree_view(const rg_ctx* c) {
    return TreeView{c->ncoarse, c->ngridmax, c->ncell, c->nx, c->ny, c->nz, c->nbound_type,
                    c->d_son, c->d_father, c->d_nbor, c->d_bound, c->d_cell_level};
}

void free_plan(rg_ctx* c, Plan& p) {
    if (p.graph) cudaGraphExecDestroy(p.graph);
    dev_free(c, p.octs);
    dev_free(c, p.icn);
    dev_free(c, p.stc);
    dev_free(c, p.kind);
    dev_free(c, p.toff);
    dev_free(c, p.tev);
    dev_free(c, p.textra);
    dev_free(c, p.xprim);
    dev_free(c, p.obox);
    dev_free(c, p.boxes);
    dev_free(c, p.read_ids);
    dev_free(c, p.lat_id);
    dev_free(c, p.lat_p);
    dev_free(c, p.bl_ext);
    dev_free(c, p.bl_off);
    dev_free(c, p.bl_brick_off);
    dev_free(c, p.tlong);
    p = Plan();
}

int rank_lists(rg_ctx* c) {
    int n = c->ngridmax;
    cudaStream_t s = c->stream;
    k_rank_init<<<nblk(n), TPB, 0, s>>>(c->d_next, n, c->d_jump, c->d_dist);
    int rounds = 1;
    while ((1LL << rounds) < (long long)n) ++rounds;
    rounds += 1;
    for (int r = 0; r < rounds; ++r) {
        k_rank_step<<<nblk(n), TPB, 0, s>>>(n, c->d_jump, c->d_dist, c->d_jump2, c->d_dist2);
        std::swap(c->d_jump, c->d_jump2);
        std::swap(c->d_dist, c->d_dist2);
    }
    k_rank_check<<<nblk(n), TPB, 0, s>>>(n, c->d_jump, c->d_dist, c->d_status);
    if (int rc = check_cuda(c, cudaGetLastError(), "list ranking")) return rc;
    c->ranked = true;
    return RG_OK;
}

int compute_cell_levels(rg_ctx* c) {
    cudaStream_t s = c->stream;
    if (int rc = check_cuda(c, cudaMemsetAsync(c->d_cell_level, 0, sizeof(int) * ((size_t)c->ncell + 1), s),
                            "memset cell_level"))
        return rc;
    k_cell_levels<<<nblk(c->ngridmax), TPB, 0, s>>>(tree_view(c), c->d_cell_level, 1 << c->params.ndim, c->d_status);
    return check_cuda(c, cudaGetLastError(), "cell levels");
}

namespace {


template <typename T>
int dalloc(rg_ctx* c, T** p, size_t n, const char* what) {
    if (dev_alloc(c, (void**)p, sizeof(T) * (n ? n : 1)) != cudaSuccess) {
        return set_error(c, RG_ERR_NOMEM, std::string("device allocation failed: ") + what);
    }
    return RG_OK;
}

template <int NDIM>
int build_plan_t(rg_ctx* c, int ilevel, Plan& P) {
    constexpr int NS = 2 * NDIM, TTD = 1 << NDIM;
    cudaStream_t s = c->stream;
    TreeView T = tree_view(c);
    free_plan(c, P);
    P.ilevel = ilevel;
    P.level0 = (ilevel == 0);
    int hv[4] = {0, 0, 0, 0};

    // ---- oct list in linked-list order
    if (!P.level0) {
        int head = 0;
        if (ilevel >= 0 && ilevel <= c->nlevelmax) head = c->h_headl[(size_t)ilevel * (c->ncpu + c->nboundary)];
        if (head > c->ngridmax || head < 0) return set_error(c, RG_ERR_TOPOLOGY, "headl entry out of range");
        if (head > 0 && c->tree_resident) {
            P.noct = c->h_numbl[(size_t)ilevel * (c->ncpu + c->nboundary)];  // checked by the count below
            if (P.noct < 1) return set_error(c, RG_ERR_TOPOLOGY, "level count and head disagree");
        } else if (head > 0) {
            int dh = 0;
            if (int rc = check_cuda(c, cudaMemcpyAsync(&dh, c->d_dist + head - 1, sizeof(int), cudaMemcpyDeviceToHost, s),
                                    "list length"))
                return rc;
            if (int rc = check_cuda(c, cudaStreamSynchronize(s), "list length sync")) return rc;
            P.noct = dh + 1;
        }
        if (P.noct == 0) {
            P.valid = true;
            return RG_OK;
        }
        if (int rc = dalloc(c, &P.octs, P.noct, "octs")) return rc;
        if (c->tree_resident) {
            // the resident tree's cached list (kept in order by the tree
            // operations, walked again only when it must be)
            const int* lo = nullptr;
            int ln = 0;
            if (int rc = level_octs_cached(c, ilevel, &lo, &ln)) return rc;
            if (ln != P.noct) return set_error(c, RG_ERR_TOPOLOGY, "level count and cached list disagree");
            cudaMemcpyAsync(P.octs, lo, sizeof(int) * (size_t)P.noct, cudaMemcpyDeviceToDevice, s);
        }
        int* d_count = c->d_scan;  // reuse scan scratch as a counter
        if (c->cap_scan < 4) {
            dev_free(c, c->d_scan);
            if (int rc = dalloc(c, &c->d_scan, 1024, "scan scratch")) return rc;
            c->cap_scan = 1024;
            d_count = c->d_scan;
        }
        if (!c->tree_resident) {
            if (!c->ranked)
                if (int rc = rank_lists(c)) return rc;
            cudaMemsetAsync(d_count, 0, 2 * sizeof(int), s);
            k_level_octs<<<nblk(c->ngridmax), TPB, 0, s>>>(c->ngridmax, c->d_jump, c->d_dist, head - 1, P.noct, P.octs,
                                                           d_count, c->d_status, false);
            cudaMemcpyAsync(&hv[0], d_count, sizeof(int), cudaMemcpyDeviceToHost, s);
            if (int rc = check_cuda(c, cudaStreamSynchronize(s), "level octs")) return rc;
            if (hv[0] != P.noct) return set_error(c, RG_ERR_TOPOLOGY, "level linked list merges with another chain");
        }
        P.ncells = P.noct * TTD;
    } else {
        P.ncells = c->ncoarse;
    }
    int nc = P.ncells;

    // ---- per-cell neighbours and interface kinds
    if (int rc = dalloc(c, &P.icn, (size_t)NS * nc, "icn")) return rc;
    if (int rc = dalloc(c, &P.stc, (size_t)NS * 2 * nc, "stencil")) return rc;
    if (int rc = dalloc(c, &P.kind, (size_t)NS * nc, "kind")) return rc;
    cudaMemsetAsync(c->d_cpos, 0xff, sizeof(int) * ((size_t)c->ncell + 1), s);
    cudaMemsetAsync(c->d_tmap, 0xff, sizeof(int) * ((size_t)c->ncell + 1), s);
    cudaMemsetAsync(c->d_pmark, 0, sizeof(int) * ((size_t)c->ncell + 1), s);
    k_plan_cpos<<<nblk(nc), TPB, 0, s>>>(T, P.octs, P.level0, P.noct, nc, c->d_cpos);
    unsigned long long* d_nact = (unsigned long long*)&c->d_status->cell_updates;
    cudaMemsetAsync(d_nact, 0, sizeof(unsigned long long), s);
    k_plan_cells<NDIM><<<nblk(nc), TPB, 0, s>>>(T, P.octs, P.level0, ilevel, P.noct, nc, c->d_cpos, P.icn, P.stc,
                                                P.kind, d_nact, c->d_status);
    if (int rc = check_cuda(c, cudaGetLastError(), "plan cells")) return rc;

    // The rest runs without a read-back: the arrays whose lengths the device
    // counts are sized by bounds, and the counts come back once at the end.
    //   extra primitives (coarser cells read by ghost stencils) and extra
    //   targets (coarser cells receiving reflux): distinct cells, <= ncell;
    //   targets: the level's cells and the extra ones, distinct, <= ncell;
    //   events: an own update and at most one reflux per face of each cell.
    const size_t ncell1 = (size_t)c->ncell + 1;
    const size_t tbound = std::min(ncell1, (size_t)nc * (NS + 1) + 1);  // targets + 1
    const size_t ebound = (size_t)nc * (NS + 1);
    int* d_nx = nullptr;  // [0] extra primitives, [1] extra targets, [2] long targets, [3] events
    int* cnt = nullptr;
    auto cleanup = [&]() { dev_free(c, d_nx); dev_free(c, cnt); };
    if (int rc = dalloc(c, &d_nx, 8, "plan counters")) return rc;
    if (int rc = dalloc(c, &cnt, tbound, "event counts")) { cleanup(); return rc; }
    if (int rc = dalloc(c, &P.xprim, ncell1, "xprim")) { cleanup(); return rc; }
    if (int rc = dalloc(c, &P.textra, ncell1, "textra")) { cleanup(); return rc; }
    if (int rc = dalloc(c, &P.toff, tbound, "toff")) { cleanup(); return rc; }
    if (int rc = dalloc(c, &P.tev, ebound, "events")) { cleanup(); return rc; }
    if (int rc = dalloc(c, &P.tlong, tbound, "long targets")) { cleanup(); return rc; }
    cudaMemsetAsync(d_nx, 0, sizeof(int) * 8, s);
    k_plan_xprim<NDIM><<<nblk(nc), TPB, 0, s>>>(nc, c->d_cpos, P.icn, P.stc, P.kind, c->d_pmark, P.xprim, d_nx);
    k_ev_claim<NDIM><<<nblk(nc), TPB, 0, s>>>(nc, c->d_cpos, P.icn, P.kind, c->d_tmap, P.textra, d_nx + 1);

    // ---- ordered event lists (CSR over targets): counts beyond the last
    //      target stay 0, so the offsets there hold the total
    cudaMemsetAsync(cnt, 0, sizeof(int) * tbound, s);
    k_ev_count<NDIM><<<nblk(nc), TPB, 0, s>>>(nc, c->d_cpos, c->d_tmap, P.icn, P.kind, cnt);
    if (int rc = exclusive_scan_dev(c, cnt, P.toff, (int)tbound, d_nx + 3)) { cleanup(); return rc; }
    cudaMemsetAsync(cnt, 0, sizeof(int) * tbound, s);
    k_ev_fill<NDIM><<<nblk(nc), TPB, 0, s>>>(nc, P.level0, P.noct, c->d_cpos, c->d_tmap, P.icn, P.kind, P.toff, cnt,
                                             P.tev);
    // long targets (more than kLongEvents events): their events are sorted a
    // block each, the rest a thread each
    k_long_targets<<<nblk((long long)tbound), TPB, 0, s>>>(nc, d_nx + 1, P.toff, kLongEvents, P.tlong, d_nx + 2);
    k_ev_sort<<<nblk((long long)tbound), TPB, 0, s>>>(nc, d_nx + 1, P.toff, P.tev, kLongEvents);
    k_ev_sort_long<<<2 * c->sm_count, kSortThreads, 0, s>>>(P.tlong, d_nx + 2, P.toff, P.tev);
    if (int rc = check_cuda(c, cudaGetLastError(), "plan events")) { cleanup(); return rc; }
    long long nact = 0;
    cudaMemcpyAsync(hv, d_nx, 4 * sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&nact, d_nact, sizeof(long long), cudaMemcpyDeviceToHost, s);
    cleanup();
    // one wait: the counts, and the device's checks (the list, the cells)
    if (int rc = check_device_status(c)) return rc;
    P.nextra_prim = hv[0];
    P.ntarg = nc + hv[1];
    P.nlong = hv[2];
    P.nevents = hv[3];
    P.nactive = nact;
    if ((size_t)P.ntarg + 1 > tbound || (size_t)P.nevents > ebound)
        return set_error(c, RG_ERR_TOPOLOGY, "plan counts above their bounds");
    P.valid = true;
    return RG_OK;
}

}  // namespace

int build_plan(rg_ctx* c, int ilevel, Plan& plan) {
    switch (c->params.ndim) {
        case 1: return build_plan_t<1>(c, ilevel, plan);
        case 3: return build_plan_t<3>(c, ilevel, plan);
        default: return set_error(c, RG_ERR_UNSUPPORTED, "ndim must be 1 or 3");
    }
}

// Exclusive scan of n ints on the context stream, the grand total left in
// device memory (*total_dev; nullptr: the scan scratch).  Enqueue only.
int exclusive_scan_dev(rg_ctx* c, const int* in, int* out, int n, int* total_dev, int** total_at) {
    int nb = (n + SCAN_ITEMS - 1) / SCAN_ITEMS;
    if (nb < 1) nb = 1;
    size_t need = (size_t)nb + 1;
    if (c->cap_scan < need) {
        dev_free(c, c->d_scan);
        c->d_scan = nullptr;
        if (dev_alloc(c, &c->d_scan, sizeof(int) * need) != cudaSuccess) return set_error(c, RG_ERR_NOMEM, "scan scratch");
        c->cap_scan = need;
    }
    int* grand = total_dev ? total_dev : c->d_scan + nb;
    k_scan_blocks<<<nb, SCAN_TPB, 0, c->stream>>>(in, out, n, c->d_scan);
    k_scan_sums<<<1, SCAN_TPB, 0, c->stream>>>(c->d_scan, nb, grand);
    k_scan_add<<<nb, SCAN_TPB, 0, c->stream>>>(out, n, c->d_scan);
    if (total_at) *total_at = grand;
    return check_cuda(c, cudaGetLastError(), "scan");
}

// Exclusive scan of n ints on the context stream; returns the grand total.
int exclusive_scan(rg_ctx* c, const int* in, int* out, int n, int* total) {
    int* grand = nullptr;
    if (int rc = exclusive_scan_dev(c, in, out, n, nullptr, &grand)) return rc;
    if (int rc = check_cuda(c, cudaMemcpyAsync(total, grand, sizeof(int), cudaMemcpyDeviceToHost, c->stream),
                            "scan total"))
        return rc;
    return check_cuda(c, cudaStreamSynchronize(c->stream), "scan sync");
}

int level_oct_list(rg_ctx* c, int ilevel, int* out, int cap, int* noct) {
    *noct = 0;
    if (ilevel < 1 || ilevel > c->nlevelmax) return set_error(c, RG_ERR_ARG, "level outside 1..nlevelmax");
    const int head = c->h_headl[(size_t)ilevel * (c->ncpu + c->nboundary)];
    if (head > c->ngridmax || head < 0) return set_error(c, RG_ERR_TOPOLOGY, "headl entry out of range");
    if (head == 0) return RG_OK;
    cudaStream_t s = c->stream;
    int dh = 0, count = 0;
    if (c->tree_resident) {
        // the resident tree keeps every level's count on the host: no read of
        // the list length (a longer list raises DE_LIST in k_level_octs, a
        // shorter one fails the count check below)
        dh = c->h_numbl[(size_t)ilevel * (c->ncpu + c->nboundary)] - 1;
        if (dh < 0) return set_error(c, RG_ERR_TOPOLOGY, "level count and head disagree");
    } else {
        if (int rc = check_cuda(c, cudaMemcpyAsync(&dh, c->d_dist + head - 1, sizeof(int), cudaMemcpyDeviceToHost, s),
                                "list length"))
            return rc;
        if (int rc = check_cuda(c, cudaStreamSynchronize(s), "list length sync")) return rc;
    }
    const int n = dh + 1;
    if (n > cap) return set_error(c, RG_ERR_TOPOLOGY, "level list longer than ngridmax");
    if (!c->ranked)
        if (int rc = rank_lists(c)) return rc;
    if (c->cap_scan < 4) {
        dev_free(c, c->d_scan);
        if (int rc = dalloc(c, &c->d_scan, 1024, "scan scratch")) return rc;
        c->cap_scan = 1024;
    }
    cudaMemsetAsync(c->d_scan, 0, 2 * sizeof(int), s);
    // with the tree resident the count is the host's own: the chain is
    // checked on the device and the host does not wait (a mismatch is
    // reported by the next call that synchronises)
    k_level_octs<<<nblk(c->ngridmax), TPB, 0, s>>>(c->ngridmax, c->d_jump, c->d_dist, head - 1, n, out, c->d_scan,
                                                   c->d_status, c->tree_resident);
    if (c->tree_resident) {
        *noct = n;
        return check_cuda(c, cudaGetLastError(), "level octs");
    }
    cudaMemcpyAsync(&count, c->d_scan, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (int rc = check_cuda(c, cudaStreamSynchronize(s), "level octs")) return rc;
    if (count != n) return set_error(c, RG_ERR_TOPOLOGY, "level linked list merges with another chain");
    *noct = n;
    return RG_OK;
}

int level_octs_cached(rg_ctx* c, int ilevel, const int** octs, int* noct) {
    *octs = nullptr;
    *noct = 0;
    if (ilevel < 1 || ilevel > c->nlevelmax) return set_error(c, RG_ERR_ARG, "level outside 1..nlevelmax");
    if (!c->tree_resident) return set_error(c, RG_ERR_STATE, "oct-list cache needs the device-resident tree");
    if (c->lvl_octs.size() < (size_t)c->nlevelmax + 1) {
        c->lvl_octs.resize((size_t)c->nlevelmax + 1, nullptr);
        c->lvl_cap.resize((size_t)c->nlevelmax + 1, 0);
        c->lvl_n.resize((size_t)c->nlevelmax + 1, 0);
        c->lvl_ver.resize((size_t)c->nlevelmax + 1, -1);
    }
    const size_t L = (size_t)ilevel;
    if (c->lvl_ver[L] == c->topo_version && !c->tree_dirty) {
        *octs = c->lvl_octs[L];
        *noct = c->lvl_n[L];
        return RG_OK;
    }
    const int n = c->h_numbl[L * (c->ncpu + c->nboundary)];
    if (n > c->lvl_cap[L]) {
        dev_free(c, c->lvl_octs[L]);
        c->lvl_octs[L] = nullptr;
        c->lvl_cap[L] = 0;
        const int cap = (n + 1023) / 1024 * 1024;
        if (int rc = check_cuda(c, dev_alloc(c, &c->lvl_octs[L], sizeof(int) * (size_t)cap), "level oct list"))
            return rc;
        c->lvl_cap[L] = cap;
    }
    int got = 0;
    if (int rc = level_oct_list(c, ilevel, c->lvl_octs[L], c->lvl_cap[L], &got)) return rc;
    c->lvl_n[L] = got;
    c->lvl_ver[L] = c->topo_version;
    *octs = c->lvl_octs[L];
    *noct = got;
    return RG_OK;
}

}  // namespace rg
