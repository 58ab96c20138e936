// Per-Gaussian kernels of the gs_b200 pipeline:
//   * stage kernels with the reference's buffer layouts (SH only,
//     projection only), used by the stage API;
//   * the fused frame kernel: SH colour + EWA projection + tile rectangle +
//     exact per-Gaussian overlap count (warp-cooperative) + single-pass
//     decoupled look-back scan of the counts into key offsets, for several
//     views per block so the SH coefficients are read once per group;
//   * the emit kernel that writes (tile|depth, index) keys at those offsets.
#include "gs_kernels.h"

namespace gs {

// ---- stage kernels (reference layouts) -------------------------------------

template <int DEG>
__global__ void __launch_bounds__(256) sh_stage_kernel(int64_t n, const float4* __restrict__ pos,
                                                       const float* __restrict__ sh, int sh_count,
                                                       const ViewParams v, float4* __restrict__ color)
{
    // The grouped SH layout is [group of 256][coefficient][256]; with one
    // Gaussian per thread and 256-thread blocks every coefficient load of a
    // warp is one contiguous 128-byte line (gaussian_render.cu:109-112).
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    const float4 p = __ldg(&pos[i]);
    const float3 d = view_dir(v, p);
    const float* base = sh + (int64_t)blockIdx.x * 256 * sh_count + threadIdx.x;
    const float3 c = sh_color<DEG>(d.x, d.y, d.z, base, 256);
    color[i] = make_float4(c.x, c.y, c.z, p.w);
}

__global__ void __launch_bounds__(256) project_stage_kernel(int64_t n, const float4* __restrict__ pos,
                                                            const float4* __restrict__ sr, const ViewParams v,
                                                            float2* __restrict__ xy, float* __restrict__ z,
                                                            float4* __restrict__ ell, float4* __restrict__ conic)
{
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    const Splat s = project_gaussian(__ldg(&pos[i]), __ldg(&sr[i]), v);
    xy[i] = make_float2(s.x, s.y);
    z[i] = s.z;
    ell[i] = make_float4(s.cs, s.sn, s.ex, s.ey);
    conic[i] = make_float4(s.ca, s.cb, s.cc, 0.0f);
}

// ---- warp-cooperative overlap counting -------------------------------------
//
// Each lane owns one Gaussian with `cand` candidate tiles.  The warp walks
// the concatenation of its 32 candidate lists 32 candidates at a time, so
// one huge splat does not serialise its lane: lane l tests candidate
// base + l of whichever Gaussian owns it (found by a 5-step search over the
// warp's inclusive scan).

struct WarpCands {
    int incl, excl, total;
};

__device__ __forceinline__ WarpCands warp_scan_cands(const int cand)
{
    const int lane = threadIdx.x & 31;
    int incl = cand;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
    }
    WarpCands w;
    w.incl = incl;
    w.excl = incl - cand;
    w.total = __shfl_sync(kFull, incl, 31);
    return w;
}

__device__ __forceinline__ int owner_of(const int incl, const int c)
{
    int pos = 0;
#pragma unroll
    for (int b = 16; b >= 1; b >>= 1) {
        const int t = __shfl_sync(kFull, incl, pos + b - 1);
        if (t <= c) pos += b;
    }
    return pos;
}

__device__ __forceinline__ unsigned lane_range_mask(const int lo, const int hi)
{
    if (hi <= lo) return 0u;
    const unsigned mhi = hi >= 32 ? kFull : ((1u << hi) - 1u);
    const unsigned mlo = (1u << lo) - 1u;
    return mhi & ~mlo;
}

// Returns this lane's number of overlapping tiles; for rectangles of at
// most 32 candidates also the hit mask (bit c = candidate c overlaps).
// With a non-null `tile_count`, every overlap also adds one to its tile's
// count (all lanes of the warp render the same view).  With `aggregate`,
// lanes that hit the same tile in one step add their number with one atomic:
// neighbouring Gaussians of a spatially ordered scene mostly share tiles,
// and when a frame has few tiles, many atomics on one address serialise.
// With many tiles the atomics spread out and the grouping costs more than
// it saves.
//
// The overlap test is the reference's, in two phases: the walk decides every
// candidate the cheap evaluation can call, and only if some candidate of the
// warp was too close to call does a second walk settle those in IEEE
// arithmetic.  Keeping the IEEE code out of the first walk keeps it free of
// register spills.
__device__ __forceinline__ void add_hits(const unsigned bal, const WarpCands& w, const int base, const int cand,
                                         const int c0, int& hits, uint32_t& mask)
{
    const unsigned bits = bal & lane_range_mask(max(w.excl - base, 0), min(w.incl - base, 32));
    if (bits) {
        hits += __popc(bits);
        if (cand <= 32) {
            // lane l of this chunk is walk index base + l - excl of its
            // owner; the walk skips the owner's centre candidate c0
            uint32_t mk = (w.excl >= base) ? (bits >> (w.excl - base)) : (bits << (base - w.excl));
            if (c0 >= 0) {
                const uint32_t low = (1u << c0) - 1u;
                mk = (mk & low) | ((mk & ~low) << 1);
            }
            mask |= mk;
        }
    }
}

// The candidate index in the owner's rectangle of walk index k: the walk
// leaves out the owner's centre candidate oc0 (counted before the walk).
__device__ __forceinline__ int walk_candidate(const int k, const int oc0) { return (oc0 >= 0 && k >= oc0) ? k + 1 : k; }

__device__ __forceinline__ int warp_count_hits(const Ell& e, const int4 r, const int cand, const ViewParams& v,
                                               uint32_t& mask, uint32_t* tile_count = nullptr,
                                               const bool aggregate = false)
{
    const int lane = threadIdx.x & 31;
    // The tile holding the centre is a hit (the centre test decides it):
    // each lane counts its own before the walk, which then leaves it out --
    // half of the candidates on the benchmark's views.  The tile is found
    // with the tile rectangle's own arithmetic and confirmed with the
    // centre test's; a centre on a tile border falls through to the walk.
    int c0 = -1, tile0 = 0;
    if (cand > 0) {
        const int gx = (int)floorf((e.cx + 1.0f) * 0.5f * v.tiles_xf);
        const int gy = (int)floorf((e.cy + 1.0f) * 0.5f * v.tiles_yf);
        const int lx = gx - r.x, ly = gy - r.y;
        if (lx >= 0 && lx < r.z && ly >= 0 && ly < r.w && gx >= 0 && gx < v.tiles_x && gy >= 0 && gy < v.tiles_y) {
            float x0, y0, x1, y1;
            tile_clip_rect(v, gx, gy, x0, y0, x1, y1);
            if (e.cx > x0 && e.cx < x1 && e.cy > y0 && e.cy < y1) {
                c0 = ly * r.z + lx;
                tile0 = gy * v.tiles_x + gx;
            }
        }
    }
    const bool pre = c0 >= 0;
    const WarpCands w = warp_scan_cands(cand - (pre ? 1 : 0));
    int hits = pre ? 1 : 0;
    mask = (pre && cand <= 32) ? (1u << c0) : 0u;
    bool undecided = false;
    {
        const unsigned bal = __ballot_sync(kFull, pre);
        if (tile_count && pre) {
            if (aggregate) {
                const unsigned grp = __match_any_sync(bal, tile0);
                if (lane == __ffs(grp) - 1) atomicAdd(&tile_count[v.tile_offset + tile0], (unsigned)__popc(grp));
            } else {
                atomicAdd(&tile_count[v.tile_offset + tile0], 1u);
            }
        }
    }
    auto owner_ell = [&](const int o, Ell& oe, int4& orr) {
        oe.cx = __shfl_sync(kFull, e.cx, o);
        oe.cy = __shfl_sync(kFull, e.cy, o);
        oe.cs = __shfl_sync(kFull, e.cs, o);
        oe.sn = __shfl_sync(kFull, e.sn, o);
        oe.ex = __shfl_sync(kFull, e.ex, o);
        oe.ey = __shfl_sync(kFull, e.ey, o);
        orr.x = __shfl_sync(kFull, r.x, o);
        orr.y = __shfl_sync(kFull, r.y, o);
        orr.z = __shfl_sync(kFull, r.z, o);
        orr.w = __shfl_sync(kFull, r.w, o);
    };
    for (int base = 0; base < w.total; base += 32) {
        const int c = base + lane;
        const int o = owner_of(w.incl, c);
        Ell oe;
        int4 orr;
        owner_ell(o, oe, orr);
        const int oexcl = __shfl_sync(kFull, w.excl, o);
        const int oc0 = __shfl_sync(kFull, c0, o);
        int st = 0;
        int tile = 0;
        if (c < w.total) st = candidate_state(oe, orr, walk_candidate(c - oexcl, oc0), v, tile);
        undecided |= st < 0;
        const bool hit = st > 0;
        const unsigned bal = __ballot_sync(kFull, hit);
        if (tile_count && hit) {
            if (aggregate) {
                const unsigned grp = __match_any_sync(bal, tile);
                if (lane == __ffs(grp) - 1) atomicAdd(&tile_count[v.tile_offset + tile], (unsigned)__popc(grp));
            } else {
                atomicAdd(&tile_count[v.tile_offset + tile], 1u);
            }
        }
        add_hits(bal, w, base, cand, c0, hits, mask);
    }
    if (__any_sync(kFull, undecided)) {
        // rare: the candidates too close to call, in IEEE arithmetic
        for (int base = 0; base < w.total; base += 32) {
            const int c = base + lane;
            const int o = owner_of(w.incl, c);
            Ell oe;
            int4 orr;
            owner_ell(o, oe, orr);
            const int oexcl = __shfl_sync(kFull, w.excl, o);
            const int oc0 = __shfl_sync(kFull, c0, o);
            int tile = 0;
            bool hit = false;
            const int oc = walk_candidate(c - oexcl, oc0);
            if (c < w.total && candidate_state(oe, orr, oc, v, tile) < 0) hit = candidate_hit_ieee(oe, tile, v);
            const unsigned bal = __ballot_sync(kFull, hit);
            if (!bal) continue;
            if (tile_count && hit) atomicAdd(&tile_count[v.tile_offset + tile], 1u);
            add_hits(bal, w, base, cand, c0, hits, mask);
        }
    }
    return hits;
}

// ---- block scan + decoupled look-back along one chain ---------------------------

// This thread's exclusive offset within a chain of blocks (`status[0..len)`,
// block `link` of it); the last block of the chain writes the chain total.
__device__ __forceinline__ int64_t chain_offsets(const int hits, uint64_t* status, const int64_t link,
                                                 const int64_t len, const uint32_t epoch, int64_t* chain_total,
                                                 int* err)
{
    __shared__ int s_warp[8];
    __shared__ int64_t s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = hits;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int k = 0; k < 8; ++k) {
            const int t = s_warp[k];
            s_warp[k] = run;
            run += t;
        }
        const uint64_t agg = (uint64_t)run;
        uint64_t excl = 0;
        if (link == 0) {
            store_status(status, status_word(kFlagP, epoch, agg));
        } else {
            store_status(status + link, status_word(kFlagA, epoch, agg));
            excl = look_back(status, link, 1, epoch, err, kErrTimeout);
            store_status(status + link, status_word(kFlagP, epoch, excl + agg));
        }
        s_base = (int64_t)excl;
        if (link == len - 1) *chain_total = (int64_t)(excl + agg);
    }
    __syncthreads();
    const int64_t r = s_base + s_warp[warp] + (incl - hits);
    __syncthreads();  // s_warp / s_base are reused by the next call
    return r;
}

__device__ __forceinline__ int64_t acquire_tile(unsigned long long* counter)
{
    __shared__ int64_t s_tile;
    if (threadIdx.x == 0) s_tile = (int64_t)atomicAdd(counter, 1ull);
    __syncthreads();
    const int64_t t = s_tile;
    return t;
}

// ---- fused frame kernel ------------------------------------------------------

//
// Block `tile` (taken in dynamic order, so a look-back only ever waits on a
// block that is already running) owns group g = tile % groups for views
// [c*vpb, (c+1)*vpb), c = tile / groups.  It reads position and
// scale/rotation of its 256 Gaussians once and, for SH scenes, brings the
// group's coefficients (the first 3*(DEG+1)^2 rows of the grouped layout,
// contiguous) into shared memory with one TMA bulk copy.  Then per view:
// SH colour, projection, tile rectangle, exact overlap count, and the
// within-view key offset from that view's look-back chain.  Gaussians that
// overlap no tile write only their offset.
//
// BUCKET: no scan at all -- each overlapping (view, Gaussian) takes a slot
// (one atomic per warp) and adds its overlaps to the per-tile counts; the
// blocks are independent and run in launch order.
// Blocks per SM: 4 (64 registers); the exact projection at SH degree 3
// keeps 80 registers (3 blocks)
template <int DEG, bool BUCKET, bool FAST>
__global__ void __launch_bounds__(256, (DEG >= 3 && !FAST) ? 3 : 4) frame_project_kernel(FrameArgs a)
{
    extern __shared__ __align__(128) float s_sh[];  // [3*(DEG+1)^2][256]
    __shared__ __align__(8) uint64_t s_bar;
    const int64_t tile = BUCKET ? (int64_t)blockIdx.x : acquire_tile(a.tile_counter);
    const int64_t chunk = tile / a.groups;
    const int64_t group = tile - chunk * a.groups;
    const int64_t i = group * 256 + threadIdx.x;
    const bool valid = i < a.n;
    const int v0 = (int)chunk * a.views_per_block;
    const int v1 = min(a.num_views, v0 + a.views_per_block);
    const uint32_t epoch = a.epoch_dev ? *a.epoch_dev : a.epoch;
    constexpr int NCOEF = DEG >= 0 ? 3 * (DEG + 1) * (DEG + 1) : 0;

    if (DEG >= 0) {
        if (threadIdx.x == 0) {
            mbar_init(&s_bar, 1);
            bulk_load(s_sh, a.sh + group * 256 * (int64_t)a.sh_count, NCOEF * 256 * sizeof(float), &s_bar);
        }
    }
    float4 p = make_float4(0.f, 0.f, 0.f, 0.f), sr = p, cin = p;
    int64_t gid = i;  // the Gaussian's caller index: equal depths are ordered by it
    if (valid) {
        if (BUCKET && a.orig) gid = __ldg(&a.orig[i]);
        p = __ldg(&a.pos[i]);
        sr = __ldg(&a.sr[i]);
        if (DEG < 0) cin = __ldg(&a.color_in[i]);
    }
    if (DEG >= 0) {
        __syncthreads();  // barrier initialised before anyone polls it
        int spins = 0;
        while (!mbar_try_wait(&s_bar, 0)) {
            if (++spins > kSpinLimit) {
                // a bulk copy from valid device memory always lands; report
                // and carry on (the frame is discarded by the host)
                if (threadIdx.x == 0) atomicCAS(a.err, 0, kErrTimeout);
                break;
            }
        }
    }

    for (int view = v0; view < v1; ++view) {
        const ViewParams& v = a.views[view];
        const int64_t o = (int64_t)view * a.n + i;
        Ell e = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        int4 r = make_int4(0, 0, 0, 0);
        int cand = 0;
        Splat s;
        float4 col = cin;
        bool projected = false;
        if (valid) {
            // outside the frustum: culled, no tile (whole warps of a
            // spatially ordered scene skip the projection together)
            const ViewPos w = view_position<FAST>(p, v);
            if (in_frustum(w)) {
                projected = true;
                s = project_gaussian<FAST>(w, sr, v);
                e = {s.x, s.y, s.cs, s.sn, s.ex, s.ey};
                r = tile_rect(e, v);
                cand = rect_candidates(r);
            }
        }
        uint32_t mask;
        // the overlap test is the reference's in every mode: the tile lists
        // of the projected floats are exactly those of the reference's build
        const int hits = warp_count_hits(e, r, cand, v, mask, BUCKET ? a.tile_count : nullptr, a.aggregate != 0);
        int64_t o_out = o;  // where this item's outputs go
        if (BUCKET) {
            const unsigned bal = __ballot_sync(kFull, hits > 0);
            if (bal == 0) continue;  // warp-uniform
            unsigned long long first = 0;
            if ((threadIdx.x & 31) == 0) first = atomicAdd(a.slot_counter, (unsigned long long)__popc(bal));
            first = __shfl_sync(kFull, first, 0);
            o_out = (int64_t)first + __popc(bal & lanemask_lt());
            if (hits > 0) a.offsets[o_out] = (int32_t)((int64_t)view * a.n + gid);
        } else {
            const int64_t off = chain_offsets(hits, a.status + (int64_t)view * a.groups, group, a.groups, epoch,
                                              a.view_total + view, a.err);
            if (valid) a.offsets[o] = (int32_t)off;
        }
        if (valid) {
            const int64_t o = o_out;
            if (a.probe_xy) {
                const int64_t q = (int64_t)view * a.n + gid;
                if (projected) {
                    a.probe_xy[q] = make_float2(s.x, s.y);
                    a.probe_z[q] = s.z;
                    a.probe_ell[q] = make_float4(s.cs, s.sn, s.ex, s.ey);
                    a.probe_conic[q] = make_float4(s.ca, s.cb, s.cc, 0.0f);
                } else {
                    a.probe_xy[q] = make_float2(-128.0f, -128.0f);
                    a.probe_z[q] = -128.0f;
                    a.probe_ell[q] = make_float4(0.f, 0.f, 0.f, 0.f);
                    a.probe_conic[q] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
            }
            if (hits > 0) {
                // the colour only matters for items that reach a tile, so the
                // SH evaluation runs after the overlap test
                if (DEG >= 0) {
                    const float3 d = view_dir(v, p);
                    const float3 c = sh_color<DEG, false>(d.x, d.y, d.z, s_sh + threadIdx.x, 256);
                    col = make_float4(c.x, c.y, c.z, p.w);
                }
                if (a.probe_color) a.probe_color[(int64_t)view * a.n + gid] = col;
                a.z[o] = s.z;
                a.rect[o] = pack_rect(r);
                a.hitmask[o] = mask;
                if (cand > 32) a.ell[o] = make_float4(s.cs, s.sn, s.ex, s.ey);
                if (a.raster_mode == 0 || cand > 32) a.xy[o] = make_float2(s.x, s.y);
                if (a.raster_mode == 0) {
                    a.color[o] = col;
                    a.conic[o] = make_float4(s.ca, s.cb, s.cc, 0.0f);
                } else {
                    float ex, ey, A = -0.72134752f * s.ca, B = -1.44269504f * s.cb, C = -0.72134752f * s.cc;
                    float L = lg2_approx(col.w);
                    const float det = s.ca * s.cc - s.cb * s.cb;
                    if (!(det > 0.0f) || !(s.ca > 0.0f) || !(s.cc > 0.0f) || !(col.w > kCullAlpha)) {
                        // contributes nothing anywhere: alpha below the cutoff,
                        // or a conic that is not positive definite
                        ex = ey = -1e30f;
                        A = B = C = 0.0f;
                        L = -1e30f;
                    } else {
                        // qc = 2 ln(opacity / cutoff) = 2 ln 2 (L + 18); 1.0001
                        // covers the approximations
                        const float qc = 1.38643f * (L + 18.0f);
                        const float rdet = rcp_approx(det);
                        ex = sqrt_approx(qc * s.cc * rdet);
                        ey = sqrt_approx(qc * s.ca * rdet);
                    }
                    a.rec[3 * o + 0] = make_float4(s.x, s.y, ex, ey);
                    a.rec[3 * o + 1] = make_float4(A, B, C, L);
                    a.rec[3 * o + 2] = make_float4(col.x, col.y, col.z, 0.0f);
                }
            }
        }
    }
}

// Count-only variant for the stage API: rectangle + exact count + scan from
// already projected (xy, ellipse) in the reference layouts (one view).
__global__ void __launch_bounds__(256) count_stage_kernel(FrameArgs a)
{
    const int64_t tile = acquire_tile(a.tile_counter);
    const int64_t i = tile * 256 + threadIdx.x;
    const bool valid = i < a.n;
    const ViewParams& v = a.views[0];
    Ell e = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int4 r = make_int4(0, 0, 0, 0);
    int cand = 0;
    if (valid) {
        const float2 c = __ldg(&a.xy[i]);
        const float4 el = __ldg(&a.ell[i]);
        e = {c.x, c.y, el.x, el.y, el.z, el.w};
        r = tile_rect(e, v);
        cand = rect_candidates(r);
        a.rect[i] = pack_rect(r);
    }
    uint32_t mask;
    const int hits = warp_count_hits(e, r, cand, v, mask);
    const int64_t off = chain_offsets(hits, a.status, tile, a.groups, a.epoch, a.view_total, a.err);
    if (valid) {
        a.offsets[i] = (int32_t)off;
        a.hitmask[i] = mask;
    }
}

__global__ void view_base_kernel(const int64_t* view_total, int num_views, int64_t* view_base, int64_t* total,
                                 int64_t capacity, int64_t* sort_n, int* overflow)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        int64_t run = 0;
        for (int v = 0; v < num_views; ++v) {
            view_base[v] = run;
            run += view_total[v];
        }
        *total = run;
        if (sort_n) {
            *sort_n = run < capacity ? run : capacity;
            *overflow = run > capacity ? 1 : 0;
        }
    }
}

// ---- emit -------------------------------------------------------------------
//
// Rewalks each warp's candidates and writes every hit at
// view_base + offsets[g] + (number of earlier hits of g), so keys leave in
// (view, Gaussian) order with tiles ascending inside a Gaussian; a stable
// sort then breaks equal keys by index.  The key holds the global tile id
// (view tile offset + tile), the value the view-flattened Gaussian index.
__global__ void __launch_bounds__(256) emit_kernel(EmitArgs a)
{
    const int64_t gi = (int64_t)blockIdx.x * 256 + threadIdx.x;  // over views * n
    const int64_t total_items = (int64_t)a.num_views * a.n;
    const bool valid = gi < total_items;
    // a warp may straddle two views; every owner's view travels with it
    const int view = valid ? (int)(gi / a.n) : 0;
    const int lane = threadIdx.x & 31;

    int cand = 0, hits = 0;
    int4 r = make_int4(0, 0, 0, 0);
    Ell e = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float depth = 0.f;
    int64_t off = 0;
    if (valid) {
        const int64_t i = gi - (int64_t)view * a.n;
        const int64_t own = a.offsets[gi];
        const int64_t next = (i + 1 < a.n) ? (int64_t)a.offsets[gi + 1] : a.view_total[view];
        hits = (int)(next - own);
        off = a.view_base[view] + own;
        if (hits > 0) {
            r = unpack_rect(a.rect[gi]);
            cand = rect_candidates(r);
            depth = a.z[gi];
            if (cand <= 32 && a.hitmask) {
                // the counting pass recorded which candidates overlap: expand
                // the mask in candidate order, no overlap test needed
                const ViewParams& v = a.views[view];
                uint32_t m = a.hitmask[gi];
                int64_t dst = off;
                while (m) {
                    const int c = __ffs(m) - 1;
                    m &= m - 1;
                    int ly, lx;
                    divmod_small(c, r.z, ly, lx);
                    const int gx = r.x + lx, gy = r.y + ly;
                    if (dst < a.capacity) {
                        a.keys[dst] = make_key((uint64_t)(v.tile_offset + gy * v.tiles_x + gx), depth);
                        a.values[dst] = (int32_t)gi;
                    }
                    ++dst;
                }
                cand = 0;  // done: stays out of the cooperative walk
            } else {
                const float2 c = a.xy[gi];
                const float4 el = a.ell[gi];
                e = {c.x, c.y, el.x, el.y, el.z, el.w};
            }
        }
    }
    // rectangles with more than 32 candidates: the warp walks them together
    if (__ballot_sync(kFull, cand > 0) == 0) return;
    const WarpCands w = warp_scan_cands(cand);
    int running = 0;
    for (int base = 0; base < w.total; base += 32) {
        const int c = base + lane;
        const int o = owner_of(w.incl, c);
        Ell oe;
        oe.cx = __shfl_sync(kFull, e.cx, o);
        oe.cy = __shfl_sync(kFull, e.cy, o);
        oe.cs = __shfl_sync(kFull, e.cs, o);
        oe.sn = __shfl_sync(kFull, e.sn, o);
        oe.ex = __shfl_sync(kFull, e.ex, o);
        oe.ey = __shfl_sync(kFull, e.ey, o);
        int4 orr;
        orr.x = __shfl_sync(kFull, r.x, o);
        orr.y = __shfl_sync(kFull, r.y, o);
        orr.z = __shfl_sync(kFull, r.z, o);
        orr.w = __shfl_sync(kFull, r.w, o);
        const int oexcl = __shfl_sync(kFull, w.excl, o);
        const int oincl = __shfl_sync(kFull, w.incl, o);
        const int orun = __shfl_sync(kFull, running, o);
        const float oz = __shfl_sync(kFull, depth, o);
        const long long ooff = __shfl_sync(kFull, (long long)off, o);
        const int oview = __shfl_sync(kFull, view, o);
        bool hit = false;
        int tile = 0;
        if (c < w.total)
            hit = candidate_hit(oe, orr, c - oexcl, a.views[oview], tile);
        const unsigned bal = __ballot_sync(kFull, hit);
        if (hit) {
            const unsigned omask = lane_range_mask(max(oexcl - base, 0), min(oincl - base, 32));
            const int rank = __popc(bal & omask & lanemask_lt());
            const int64_t dst = ooff + orun + rank;
            if (dst < a.capacity) {
                const int64_t gtile = a.views[oview].tile_offset + tile;
                a.keys[dst] = make_key((uint64_t)gtile, oz);
                a.values[dst] = (int32_t)((int64_t)blockIdx.x * 256 + (threadIdx.x & ~31) + o);
            }
        }
        running += __popc(bal & lane_range_mask(max(w.excl - base, 0), min(w.incl - base, 32)));
    }
}

// ---- launchers ----------------------------------------------------------------

void launch_sh_stage(int64_t n, const float4* pos, const float* sh, int sh_count, int deg, const ViewParams& v,
                     float4* color, cudaStream_t st)
{
    const unsigned grid = (unsigned)((n + 255) / 256);
    if (grid == 0) return;
    switch (deg) {
        case 0: sh_stage_kernel<0><<<grid, 256, 0, st>>>(n, pos, sh, sh_count, v, color); break;
        case 1: sh_stage_kernel<1><<<grid, 256, 0, st>>>(n, pos, sh, sh_count, v, color); break;
        case 2: sh_stage_kernel<2><<<grid, 256, 0, st>>>(n, pos, sh, sh_count, v, color); break;
        default: sh_stage_kernel<3><<<grid, 256, 0, st>>>(n, pos, sh, sh_count, v, color); break;
    }
}

void launch_project_stage(int64_t n, const float4* pos, const float4* sr, const ViewParams& v, float2* xy,
                          float* z, float4* ell, float4* conic, cudaStream_t st)
{
    const unsigned grid = (unsigned)((n + 255) / 256);
    if (grid == 0) return;
    project_stage_kernel<<<grid, 256, 0, st>>>(n, pos, sr, v, xy, z, ell, conic);
}

template <int DEG, bool BUCKET, bool FAST>
static void launch_frame_deg(const FrameArgs& a, cudaStream_t st)
{
    constexpr int NCOEF = DEG >= 0 ? 3 * (DEG + 1) * (DEG + 1) : 0;
    constexpr int smem = NCOEF * 256 * (int)sizeof(float);
    static PerDeviceOnce attr;
    attr.run([] {
        cudaFuncSetAttribute(frame_project_kernel<DEG, BUCKET, FAST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem);
    });
    frame_project_kernel<DEG, BUCKET, FAST><<<(unsigned)a.num_tiles, 256, smem, st>>>(a);
}

template <bool BUCKET, bool FAST>
static void launch_frame_mode(const FrameArgs& a, int deg, cudaStream_t st)
{
    switch (deg) {
        case -1: launch_frame_deg<-1, BUCKET, FAST>(a, st); break;
        case 0: launch_frame_deg<0, BUCKET, FAST>(a, st); break;
        case 1: launch_frame_deg<1, BUCKET, FAST>(a, st); break;
        case 2: launch_frame_deg<2, BUCKET, FAST>(a, st); break;
        default: launch_frame_deg<3, BUCKET, FAST>(a, st); break;
    }
}

// T_min frames (raster records) project with the approximate arithmetic,
// reference-compatible frames with the exact one, in both orderings.
void launch_frame_project(const FrameArgs& a, int deg, cudaStream_t st, bool bucket)
{
    if (a.num_tiles == 0) return;
    const bool fast = a.raster_mode != 0;
    if (bucket && fast)
        launch_frame_mode<true, true>(a, deg, st);
    else if (bucket)
        launch_frame_mode<true, false>(a, deg, st);
    else if (fast)
        launch_frame_mode<false, true>(a, deg, st);
    else
        launch_frame_mode<false, false>(a, deg, st);
}

void launch_count_stage(const FrameArgs& a, cudaStream_t st)
{
    const unsigned grid = (unsigned)a.num_tiles;
    if (grid == 0) return;
    count_stage_kernel<<<grid, 256, 0, st>>>(a);
}

void launch_view_base(const int64_t* view_total, int num_views, int64_t* view_base, int64_t* total, cudaStream_t st,
                      int64_t capacity, int64_t* sort_n, int* overflow)
{
    view_base_kernel<<<1, 32, 0, st>>>(view_total, num_views, view_base, total, capacity, sort_n, overflow);
}

void launch_emit(const EmitArgs& a, cudaStream_t st)
{
    const int64_t items = (int64_t)a.num_views * a.n;
    const unsigned grid = (unsigned)((items + 255) / 256);
    if (grid == 0) return;
    emit_kernel<<<grid, 256, 0, st>>>(a);
}

}  // namespace gs
