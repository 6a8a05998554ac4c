// Resident deletion index and its serving loop (no counterpart in the reference, which only runs
// whole offline searches; this is the query form of the same search).
//
// An index holds, in HBM, every deletion variant (at most max_distance <= 2 deletions) of the
// first 18 residues of n reference sequences as one sorted array of 8-byte records:
//     [ top hash bits | deletion count (2 bits) | sequence id (id_bits) ]
// sorted by hash, then deletion count, plus a directory of the first record of every value of
// the top B hash bits. A query batch at distance d <= max_distance hashes its own <= d-deletion
// variants, finds the equal-hash records whose deletion count is <= d, and verifies the
// resulting (index, query) pairs on the full strings. The answer equals what the offline search
// returns on (index sequences followed by the batch), restricted to pairs with one index row
// x and one batch row y: pairs (x, n_index + q) in (x, y) order with the reference distance.
// (Two sequences within distance d share a variant with at most d deletions on each side; the
// deletion count of a variant is fixed by its length, so the filter is exact.)
//
// This file is included by xtn_engine.cu and uses its context, buffers and primitives.

namespace xtn {

constexpr int kIndexDirBitsMax = 24;

// Variant records of index sequences: (hash & hash_mask) | deletions << id_bits | id.
struct IndexRecEmitter {
    const uint64_t* tab;
    uint64_t c1, s1, kp, hash_mask, low;
    int idbits;
    uint64_t* out;
    uint64_t o;
    __device__ IndexRecEmitter(const uint64_t* t, uint64_t* dst, uint64_t pos, uint64_t id, int ib)
        : tab(t), kp(0), low(id), idbits(ib), out(dst), o(pos) {
        const uint64_t PL = t[kTabKey];
        c1 = kPolyRI2 * PL;
        s1 = (kPolyRI - kPolyRI2) * PL;
        hash_mask = ~((1ull << (ib + 2)) - 1ull);
    }
    __device__ void put(uint64_t h, uint64_t del) { out[o++] = (h & hash_mask) | (del << idbits) | low; }
    __device__ void key(int) { put(hash_fin(tab[kTabKey]), 0); }
    __device__ void run(int p) { kp = kPolyR * tab[kTabG + p] + c1; }
    __device__ void single(int) { put(hash_fin(kp + s1), 1); }
    __device__ void pair(int, int q) { put(hash_fin(kp + tab[kTabG + q]), 2); }
};

__global__ void k_index_gen(const uint8_t* __restrict__ klen, const uint64_t* __restrict__ runinfo,
                            const uint64_t* __restrict__ tab, const uint64_t* __restrict__ voff, int n, int dmax,
                            int idbits, uint64_t* __restrict__ recs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    IndexRecEmitter e(tab + (size_t)i * kTabLen, recs, voff[i], (uint64_t)i, idbits);
    seq_items(klen[i], runinfo[i], dmax, e);
}

// dir[b] = first record whose top B bits are >= b, for b = 0 .. 2^B (dir[2^B] = V).
__global__ void k_index_dir(const uint64_t* __restrict__ recs, int64_t V, int B, uint32_t* __restrict__ dir) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > V) return;
    const int64_t cur = i < V ? (int64_t)(recs[i] >> (64 - B)) : (int64_t(1) << B);
    const int64_t prev = i > 0 ? (int64_t)(recs[i - 1] >> (64 - B)) : -1;
    for (int64_t b = prev + 1; b <= cur; b++) dir[b] = (uint32_t)i;
}

// Query variants: full 64-bit hash and the batch row of each.
struct QueryHashEmitter {
    const uint64_t* tab;
    uint64_t c1, s1, kp;
    uint64_t* qh;
    uint32_t* qrow;
    uint64_t o;
    uint32_t row;
    __device__ QueryHashEmitter(const uint64_t* t, uint64_t* h, uint32_t* r, uint64_t pos, uint32_t rw)
        : tab(t), kp(0), qh(h), qrow(r), o(pos), row(rw) {
        const uint64_t PL = t[kTabKey];
        c1 = kPolyRI2 * PL;
        s1 = (kPolyRI - kPolyRI2) * PL;
    }
    __device__ void put(uint64_t h) {
        qh[o] = h;
        qrow[o] = row;
        o++;
    }
    __device__ void key(int) { put(hash_fin(tab[kTabKey])); }
    __device__ void run(int p) { kp = kPolyR * tab[kTabG + p] + c1; }
    __device__ void single(int) { put(hash_fin(kp + s1)); }
    __device__ void pair(int, int q) { put(hash_fin(kp + tab[kTabG + q])); }
};

__global__ void k_query_gen(const uint8_t* __restrict__ klen, const uint64_t* __restrict__ runinfo,
                            const uint64_t* __restrict__ tab, const uint64_t* __restrict__ voff, int n, int d,
                            uint64_t* __restrict__ qh, uint32_t* __restrict__ qrow) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    QueryHashEmitter e(tab + (size_t)i * kTabLen, qh, qrow, voff[i], (uint32_t)i);
    seq_items(klen[i], runinfo[i], d, e);
}

// For each query variant: the index records with its hash and at most d deletions, as the
// range [lb, lb + cnt) of the sorted records.
__global__ void k_query_count(const uint64_t* __restrict__ qh, int64_t Vq, const uint64_t* __restrict__ recs,
                              const uint32_t* __restrict__ dir, int B, int idbits, int d, uint32_t* __restrict__ lb,
                              uint32_t* __restrict__ cnt) {
    int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= Vq) return;
    const uint64_t h = qh[r];
    const uint64_t b = h >> (64 - B);
    const uint64_t lo_key = (h >> (idbits + 2)) << 2;  // (hash bits, deletions 0)
    const uint64_t hi_key = lo_key | (uint64_t)d;      // (hash bits, deletions d)
    uint32_t lo = dir[b], hi = dir[b + 1];
    // first record with key >= lo_key
    uint32_t a = lo, z = hi;
    while (a < z) {
        const uint32_t m = (a + z) >> 1;
        if ((recs[m] >> idbits) < lo_key) a = m + 1;
        else z = m;
    }
    // runs of equal hash are short: walk to the end of the (hash, deletions <= d) range
    const uint32_t first = a;
    while (a < hi && (recs[a] >> idbits) <= hi_key) a++;
    lb[r] = first;
    cnt[r] = a - first;
}

__global__ void k_query_emit(const uint32_t* __restrict__ qrow, int64_t Vq, const uint64_t* __restrict__ recs,
                             const uint32_t* __restrict__ lb, const uint32_t* __restrict__ cnt,
                             const uint64_t* __restrict__ coff, int idbits, int qbits, uint64_t* __restrict__ pairs) {
    int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= Vq) return;
    const uint64_t idmask = (1ull << idbits) - 1ull;
    const uint64_t q = qrow[r];
    uint64_t o = coff[r];
    const uint32_t s = lb[r], e = s + cnt[r];
    for (uint32_t k = s; k < e; k++) pairs[o++] = ((recs[k] & idmask) << qbits) | q;
}

// Unique (index row, query row) pairs, verified on the full strings of the two stores. As in
// k_verify, each warp lists the first of each run of equal pairs among its kVerifyPer * 32
// candidates and spreads them over its lanes; repeats get distance 0 and are not kept.
__global__ void __launch_bounds__(kThreads) k_query_verify(const uint64_t* __restrict__ pairs, int64_t P, int qbits,
                                                           const uint8_t* __restrict__ ichars,
                                                           const uint32_t* __restrict__ ioffs,
                                                           const uint8_t* __restrict__ qchars,
                                                           const uint32_t* __restrict__ qoffs, int d, int measure,
                                                           int8_t* __restrict__ dist, uint8_t* __restrict__ flag) {
    __shared__ uint64_t s_pair[kVerifyWarps][32 * kVerifyPer];
    __shared__ uint8_t s_slot[kVerifyWarps][32 * kVerifyPer];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t base = ((int64_t)blockIdx.x * kVerifyWarps + warp) * (32 * kVerifyPer);
    if (base >= P) return;  // whole warp
    const unsigned lt = (1u << lane) - 1u;
    uint64_t carry = base > 0 ? pairs[base - 1] : 0ull;
    uint32_t n_work = 0;
#pragma unroll
    for (int k = 0; k < kVerifyPer; k++) {
        const int64_t i = base + k * 32 + lane;
        const bool in = i < P;
        const uint64_t p = in ? pairs[i] : 0ull;
        uint64_t prev = __shfl_up_sync(0xffffffffu, p, 1);
        if (lane == 0) prev = carry;
        carry = __shfl_sync(0xffffffffu, p, 31);
        const bool need = in && (i == 0 || prev != p);
        const unsigned mask = __ballot_sync(0xffffffffu, need);
        if (need) {
            const uint32_t w = n_work + __popc(mask & lt);
            s_pair[warp][w] = p;
            s_slot[warp][w] = (uint8_t)(k * 32 + lane);
        } else if (in) {
            dist[i] = 0;
            flag[i] = 0;
        }
        n_work += __popc(mask);
    }
    __syncwarp();
    for (uint32_t w = lane; w < n_work; w += 32) {
        const uint64_t p = s_pair[warp][w];
        const int64_t i = base + s_slot[warp][w];
        const uint32_t x = (uint32_t)(p >> qbits), y = (uint32_t)(p & ((1ull << qbits) - 1ull));
        const uint32_t sa = ioffs[x], sb = qoffs[y];
        bool keep = false;
        const int dv = pair_distance(ichars + sa, (int)(ioffs[x + 1] - sa), qchars + sb, (int)(qoffs[y + 1] - sb), d,
                                     measure, &keep);
        dist[i] = (int8_t)dv;
        flag[i] = keep ? 1 : 0;
    }
}

__global__ void k_query_compact(const uint64_t* __restrict__ pairs, int64_t P, int qbits, int n_index,
                                const int8_t* __restrict__ dist, const uint8_t* __restrict__ flag,
                                const uint32_t* __restrict__ pos, xtn_int2* __restrict__ out,
                                int8_t* __restrict__ out_dist) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P || !flag[i]) return;
    const uint64_t p = pairs[i];
    const uint32_t o = pos[i];
    out[o] = xtn_int2{(int32_t)(p >> qbits), n_index + (int32_t)(p & ((1ull << qbits) - 1ull))};
    out_dist[o] = dist[i];
}

}  // namespace xtn

// Query scratch of one serving slot (a slot also has its own context: stream, search scratch
// and result buffers).
struct xtn_query_bufs {
    DevBuf qh, qrow, qlb, qcnt, qcoff;
};

struct xtn_index {
    xtn_context* c = nullptr;  // stream, scratch and the query result buffers
    int n = 0, dmax = 0, idbits = 0, dir_bits = 0;
    uint64_t V = 0;
    DevBuf chars, offs, recs, dir;
    xtn_query_bufs qb;
    double ms_build = 0;
};

namespace xtn {

static int index_build(xtn_index* ix, int n, int dmax, bool validate) {
    xtn_context* c = ix->c;
    cudaStream_t s = c->stream;
    cudaEvent_t e0 = c->ev[0], e1 = c->ev[1];
    XTN_CK(cudaEventRecord(e0, s));
    ix->n = n;
    ix->dmax = dmax;
    ix->idbits = id_bits_for(n);
    if (ix->idbits + 2 + 16 > 64) {
        set_err("index too large");
        return XTN_ERR_LIMIT;
    }
    const uint8_t* chars = P<uint8_t>(ix->chars);
    const uint32_t* offs = P<uint32_t>(ix->offs);
    XTN_TRY(ensure(c->keys, sizeof(u128) * n));
    XTN_TRY(ensure(c->klen, (size_t)n));
    XTN_TRY(ensure(c->vcnt, sizeof(uint32_t) * n));
    XTN_TRY(ensure(c->voff, sizeof(uint64_t) * (n + 1)));
    XTN_TRY(ensure(c->runinfo, sizeof(uint64_t) * n));
    XTN_TRY(ensure(c->ktab, sizeof(uint64_t) * kTabLen * (size_t)n));
    if (validate) XTN_TRY(launch_length_check(c, offs, nullptr, n));
    XTN_LAUNCH("index_pack", k_pack<<<blocks_for(n, kPackThreads), kPackThreads, 0, s>>>(
                                 chars, offs, nullptr, n, dmax, P<u128>(c->keys), P<uint8_t>(c->klen),
                                 P<uint32_t>(c->vcnt), P<uint64_t>(c->runinfo), P<uint64_t>(c->ktab)));
    XTN_CK(cudaGetLastError());
    XTN_TRY(scan_u32_to_u64(c, P<uint32_t>(c->vcnt), P<uint64_t>(c->voff), n));
    uint64_t V = 0;
    if (validate) XTN_CK(cudaMemcpyAsync(c->h_scalar + 1, c->lencheck.p, 4, cudaMemcpyDeviceToHost, s));
    XTN_TRY(read_scalar(c, P<uint64_t>(c->voff) + n, 8, &V));
    if (validate) XTN_TRY(length_check_result(c, (uint32_t)c->h_scalar[1]));
    if (V >= (uint64_t)UINT32_MAX) {
        set_err("index has too many deletion variants (" + std::to_string(V) + ")");
        return XTN_ERR_LIMIT;
    }
    ix->V = V;
    XTN_TRY(ensure(ix->recs, sizeof(uint64_t) * V + 64));
    XTN_TRY(ensure(c->recB, sizeof(uint64_t) * V + 64));
    XTN_LAUNCH("index_gen", k_index_gen<<<blocks_for(n), kThreads, 0, s>>>(
                                P<uint8_t>(c->klen), P<uint64_t>(c->runinfo), P<uint64_t>(c->ktab),
                                P<uint64_t>(c->voff), n, dmax, ix->idbits, P<uint64_t>(ix->recs)));
    XTN_CK(cudaGetLastError());
    uint64_t* sorted = nullptr;
    XTN_TRY(sort_u64(c, ix->recs, c->recB, (int64_t)V, ix->idbits, 64, &sorted, XTN_SORT_NAMES("index_sort")));
    if (sorted != P<uint64_t>(ix->recs))
        XTN_CK(cudaMemcpyAsync(ix->recs.p, sorted, sizeof(uint64_t) * V, cudaMemcpyDeviceToDevice, s));
    int B = 1;
    while (B < kIndexDirBitsMax && (V >> (B + 3)) > 0) B++;
    B = std::min(B, 64 - ix->idbits - 2);
    ix->dir_bits = B;
    XTN_TRY(ensure(ix->dir, sizeof(uint32_t) * ((size_t(1) << B) + 1)));
    XTN_LAUNCH("index_dir", k_index_dir<<<blocks_for((int64_t)V + 1), kThreads, 0, s>>>(P<uint64_t>(ix->recs),
                                                                                        (int64_t)V, B,
                                                                                        P<uint32_t>(ix->dir)));
    XTN_CK(cudaGetLastError());
    XTN_CK(cudaEventRecord(e1, s));
    XTN_CK(cudaStreamSynchronize(s));
    XTN_TRY(check_err_word(c));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    ix->ms_build = ms;
    // the build's scratch is not needed by queries
    DevBuf* tmp[] = {&c->recB, &c->keys, &c->ktab, &c->scratch32, &c->os_status};
    for (DevBuf* b : tmp) release(*b);
    return XTN_SUCCESS;
}

// One query batch on device inputs; the result (pairs (index row, n_index + query row), int8
// distances) is left in the context's output buffers, c->n_out entries.
static int index_query(xtn_index* ix, xtn_context* c, xtn_query_bufs& qb, const uint8_t* qchars,
                       const uint32_t* qoffs, int nq, int d, int measure, bool validate) {
    cudaStream_t s = c->stream;
    c->stats = xtn_stats{};
    c->stats.n_seqs = nq;
    c->overlap_result = false;
    if (d > ix->dmax) {
        set_err("query distance " + std::to_string(d) + " exceeds the index's maximum distance " +
                std::to_string(ix->dmax));
        return XTN_ERR_ARG;
    }
    XTN_TRY(ensure(c->keys, sizeof(u128) * nq));
    XTN_TRY(ensure(c->klen, (size_t)nq));
    XTN_TRY(ensure(c->vcnt, sizeof(uint32_t) * nq));
    XTN_TRY(ensure(c->voff, sizeof(uint64_t) * (nq + 1)));
    XTN_TRY(ensure(c->runinfo, sizeof(uint64_t) * nq));
    XTN_TRY(ensure(c->ktab, sizeof(uint64_t) * kTabLen * (size_t)nq));
    if (validate) XTN_TRY(launch_length_check(c, qoffs, nullptr, nq));
    XTN_LAUNCH("query_pack", k_pack<<<blocks_for(nq, kPackThreads), kPackThreads, 0, s>>>(
                                 qchars, qoffs, nullptr, nq, d, P<u128>(c->keys), P<uint8_t>(c->klen),
                                 P<uint32_t>(c->vcnt), P<uint64_t>(c->runinfo), P<uint64_t>(c->ktab)));
    XTN_CK(cudaGetLastError());
    XTN_TRY(scan_u32_to_u64(c, P<uint32_t>(c->vcnt), P<uint64_t>(c->voff), nq));
    uint64_t Vq = 0;
    if (validate) XTN_CK(cudaMemcpyAsync(c->h_scalar + 1, c->lencheck.p, 4, cudaMemcpyDeviceToHost, s));
    XTN_TRY(read_scalar(c, P<uint64_t>(c->voff) + nq, 8, &Vq));
    if (validate) XTN_TRY(length_check_result(c, (uint32_t)c->h_scalar[1]));
    c->stats.n_variants = (int64_t)Vq;
    XTN_TRY(ensure(qb.qh, sizeof(uint64_t) * Vq));
    XTN_TRY(ensure(qb.qrow, sizeof(uint32_t) * Vq));
    XTN_TRY(ensure(qb.qlb, sizeof(uint32_t) * Vq));
    XTN_TRY(ensure(qb.qcnt, sizeof(uint32_t) * Vq));
    XTN_TRY(ensure(qb.qcoff, sizeof(uint64_t) * (Vq + 1)));
    XTN_LAUNCH("query_gen", k_query_gen<<<blocks_for(nq), kThreads, 0, s>>>(
                                P<uint8_t>(c->klen), P<uint64_t>(c->runinfo), P<uint64_t>(c->ktab),
                                P<uint64_t>(c->voff), nq, d, P<uint64_t>(qb.qh), P<uint32_t>(qb.qrow)));
    XTN_LAUNCH("query_count", k_query_count<<<blocks_for((int64_t)Vq), kThreads, 0, s>>>(
                                  P<uint64_t>(qb.qh), (int64_t)Vq, P<uint64_t>(ix->recs), P<uint32_t>(ix->dir),
                                  ix->dir_bits, ix->idbits, d, P<uint32_t>(qb.qlb), P<uint32_t>(qb.qcnt)));
    XTN_CK(cudaGetLastError());
    XTN_TRY(scan_u32_to_u64(c, P<uint32_t>(qb.qcnt), P<uint64_t>(qb.qcoff), (int64_t)Vq));
    uint64_t Pc = 0;
    XTN_TRY(read_scalar(c, P<uint64_t>(qb.qcoff) + Vq, 8, &Pc));
    c->stats.n_candidates = (int64_t)Pc;
    const int qbits = id_bits_for(nq);
    if (Pc >= (uint64_t)UINT32_MAX || ix->idbits + qbits > 64) {
        set_err("query batch too large for one round (" + std::to_string(Pc) + " candidates)");
        return XTN_ERR_LIMIT;
    }
    uint64_t nout = 0;
    if (Pc > 0) {
        XTN_TRY(ensure(c->pairA, sizeof(uint64_t) * Pc + 64));
        XTN_TRY(ensure(c->pairB, sizeof(uint64_t) * Pc + 64));
        XTN_LAUNCH("query_emit", k_query_emit<<<blocks_for((int64_t)Vq), kThreads, 0, s>>>(
                                     P<uint32_t>(qb.qrow), (int64_t)Vq, P<uint64_t>(ix->recs), P<uint32_t>(qb.qlb),
                                     P<uint32_t>(qb.qcnt), P<uint64_t>(qb.qcoff), ix->idbits, qbits,
                                     P<uint64_t>(c->pairA)));
        XTN_CK(cudaGetLastError());
        uint64_t* pairs = P<uint64_t>(c->pairA);
        if (Pc > 1)
            XTN_TRY(sort_u64(c, c->pairA, c->pairB, (int64_t)Pc, 0, ix->idbits + qbits, &pairs, XTN_SORT_NAMES("pair_sort")));
        XTN_TRY(ensure(c->dist, Pc));
        XTN_TRY(ensure(c->flag, Pc));
        XTN_TRY(ensure(c->fpos, sizeof(uint32_t) * (Pc + 1)));
        XTN_TRY(ensure(c->scratch32, sizeof(uint32_t) * scan_scratch_elems((int64_t)Pc)));
        XTN_LAUNCH("query_verify", k_query_verify<<<blocks_for((int64_t)Pc, kThreads * kVerifyPer), kThreads, 0, s>>>(
                                       pairs, (int64_t)Pc, qbits, P<uint8_t>(ix->chars), P<uint32_t>(ix->offs), qchars,
                                       qoffs, d, measure, P<int8_t>(c->dist), P<uint8_t>(c->flag)));
        XTN_TRY((scan_1p<uint8_t, uint32_t>(c, P<uint8_t>(c->flag), P<uint32_t>(c->fpos), (int64_t)Pc)));
        XTN_TRY(read_scalar(c, P<uint32_t>(c->fpos) + Pc, 4, &nout));
        XTN_TRY(ensure(c->out_pairs, sizeof(xtn_int2) * (nout + 1)));
        XTN_TRY(ensure(c->out_dist, nout + 1));
        if (nout > 0)
            XTN_LAUNCH("query_compact", k_query_compact<<<blocks_for((int64_t)Pc), kThreads, 0, s>>>(
                                            pairs, (int64_t)Pc, qbits, ix->n, P<int8_t>(c->dist), P<uint8_t>(c->flag),
                                            P<uint32_t>(c->fpos), P<xtn_int2>(c->out_pairs),
                                            P<int8_t>(c->out_dist)));
        XTN_CK(cudaGetLastError());
    }
    if (c->dev_err.p) XTN_CK(cudaMemcpyAsync(c->h_scalar + 7, c->dev_err.p, 8, cudaMemcpyDeviceToHost, s));
    XTN_CK(cudaStreamSynchronize(s));
    if (c->dev_err.p && (uint32_t)c->h_scalar[7] != 0) {
        XTN_CK(cudaMemsetAsync(c->dev_err.p, 0, 16, s));
        set_err("radix sort: a look-back wait did not complete in time");
        return XTN_ERR_CUDA;
    }
    c->n_out = (int64_t)nout;
    c->stats.n_out = (int64_t)nout;
    return XTN_SUCCESS;
}

// Grows the query buffers for a batch of nq sequences with `chars` residues at distance d, so
// that a serving loop does not reallocate device memory between requests (candidate buffers
// are sized for one candidate per query variant and grow if a batch needs more).
constexpr int kMaxServeSlots = 8;

static int index_reserve(xtn_context* c, xtn_query_bufs& qb, int64_t nq, int64_t chars, int d) {
    const int64_t Vq = nq * (d >= 2 ? 172 : 19);
    XTN_TRY(ensure(c->chars, (size_t)chars + 16));
    XTN_TRY(ensure(c->offs, sizeof(uint32_t) * (nq + 1)));
    XTN_TRY(ensure(c->keys, sizeof(u128) * nq));
    XTN_TRY(ensure(c->klen, (size_t)nq));
    XTN_TRY(ensure(c->vcnt, sizeof(uint32_t) * nq));
    XTN_TRY(ensure(c->voff, sizeof(uint64_t) * (nq + 1)));
    XTN_TRY(ensure(c->runinfo, sizeof(uint64_t) * nq));
    XTN_TRY(ensure(c->ktab, sizeof(uint64_t) * kTabLen * (size_t)nq));
    XTN_TRY(ensure(c->scratch64, sizeof(uint64_t) * scan_scratch_elems(Vq + 1)));
    XTN_TRY(ensure(qb.qh, sizeof(uint64_t) * Vq));
    XTN_TRY(ensure(qb.qrow, sizeof(uint32_t) * Vq));
    XTN_TRY(ensure(qb.qlb, sizeof(uint32_t) * Vq));
    XTN_TRY(ensure(qb.qcnt, sizeof(uint32_t) * Vq));
    XTN_TRY(ensure(qb.qcoff, sizeof(uint64_t) * (Vq + 1)));
    XTN_TRY(ensure(c->pairA, sizeof(uint64_t) * Vq + 64));
    XTN_TRY(ensure(c->pairB, sizeof(uint64_t) * Vq + 64));
    XTN_TRY(ensure(c->dist, (size_t)Vq));
    XTN_TRY(ensure(c->flag, (size_t)Vq));
    XTN_TRY(ensure(c->fpos, sizeof(uint32_t) * (Vq + 1)));
    XTN_TRY(ensure(c->scratch32, sizeof(uint32_t) * std::max(radix_scratch_elems(Vq), scan_scratch_elems(Vq))));
    XTN_TRY(ensure(c->out_pairs, sizeof(xtn_int2) * (size_t)Vq / 4 + 16));
    XTN_TRY(ensure(c->out_dist, (size_t)Vq / 4 + 16));
    return XTN_SUCCESS;
}

static int index_create_common(int device, int dmax, xtn_index** out, xtn_index** ix) {
    if (!out) {
        set_err("null output pointer");
        return XTN_ERR_ARG;
    }
    *out = nullptr;
    if (dmax < 1 || dmax > 2) {
        set_err("index maximum distance must be 1 or 2");
        return XTN_ERR_ARG;
    }
    xtn_context* c = nullptr;
    XTN_TRY(xtn_context_create(device, &c));
    *ix = new xtn_index();
    (*ix)->c = c;
    return XTN_SUCCESS;
}

static void index_free(xtn_index* ix) {
    if (!ix) return;
    if (ix->c) {
        cudaSetDevice(ix->c->device);
        cudaStreamSynchronize(ix->c->stream);
        DevBuf* bufs[] = {&ix->chars, &ix->offs, &ix->recs, &ix->dir, &ix->qb.qh, &ix->qb.qrow, &ix->qb.qlb,
                          &ix->qb.qcnt, &ix->qb.qcoff};
        for (DevBuf* b : bufs) release(*b);
        xtn_context_destroy(ix->c);
    }
    delete ix;
}

static double now_s() {
    using clk = std::chrono::steady_clock;
    static const clk::time_point t0 = clk::now();
    return std::chrono::duration<double>(clk::now() - t0).count();
}

// Bytes of device memory a query sequence may need at distance d (variant hashes, rows,
// lookup ranges and offsets, about four candidate pairs per variant with their sort buffer,
// distances and flags), used to admit batches by free memory.
static size_t query_bytes_per_seq(int d) {
    const size_t variants = d >= 2 ? 172 : 19;
    return 600 + variants * (8 + 4 + 4 + 4 + 8 + 4 * (16 + 1 + 1 + 4));
}

}  // namespace xtn

extern "C" {

int xtn_index_create(int device, const char* seqs, const uint32_t* offsets, int32_t n_seqs, int32_t max_distance,
                     xtn_index** out) {
    if (!seqs || !offsets || n_seqs < 1) {
        set_err("invalid arguments");
        if (out) *out = nullptr;
        return XTN_ERR_ARG;
    }
    xtn_index* ix = nullptr;
    XTN_TRY(index_create_common(device, max_distance, out, &ix));
    int r = check_offsets(offsets, n_seqs);
    if (r == XTN_SUCCESS) {
        const size_t nch = offsets[n_seqs];
        r = ensure(ix->chars, nch + 16);
        if (r == XTN_SUCCESS) r = ensure(ix->offs, sizeof(uint32_t) * (n_seqs + 1));
        if (r == XTN_SUCCESS &&
            (cudaMemcpyAsync(ix->chars.p, seqs, nch, cudaMemcpyHostToDevice, ix->c->stream) != cudaSuccess ||
             cudaMemcpyAsync(ix->offs.p, offsets, sizeof(uint32_t) * (n_seqs + 1), cudaMemcpyHostToDevice,
                             ix->c->stream) != cudaSuccess)) {
            set_err("index upload failed");
            r = XTN_ERR_CUDA;
        }
    }
    if (r == XTN_SUCCESS) {
        begin_run(ix->c);
        r = index_build(ix, n_seqs, max_distance, false);
        end_run(ix->c);
    }
    if (r != XTN_SUCCESS) {
        index_free(ix);
        return r;
    }
    *out = ix;
    return XTN_SUCCESS;
}

int xtn_index_create_device(int device, const char* d_seqs, const uint32_t* d_offsets, int32_t n_seqs,
                            int32_t max_distance, xtn_index** out) {
    if (!d_seqs || !d_offsets || n_seqs < 1) {
        set_err("invalid arguments");
        if (out) *out = nullptr;
        return XTN_ERR_ARG;
    }
    xtn_index* ix = nullptr;
    XTN_TRY(index_create_common(device, max_distance, out, &ix));
    int r = XTN_SUCCESS;
    uint32_t nch = 0;
    if (cudaMemcpy(&nch, d_offsets + n_seqs, sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_err("cannot read the offsets");
        r = XTN_ERR_CUDA;
    }
    if (r == XTN_SUCCESS) r = ensure(ix->chars, (size_t)nch + 16);
    if (r == XTN_SUCCESS) r = ensure(ix->offs, sizeof(uint32_t) * (n_seqs + 1));
    if (r == XTN_SUCCESS &&
        (cudaMemcpyAsync(ix->chars.p, d_seqs, nch, cudaMemcpyDeviceToDevice, ix->c->stream) != cudaSuccess ||
         cudaMemcpyAsync(ix->offs.p, d_offsets, sizeof(uint32_t) * (n_seqs + 1), cudaMemcpyDeviceToDevice,
                         ix->c->stream) != cudaSuccess)) {
        set_err("index copy failed");
        r = XTN_ERR_CUDA;
    }
    if (r == XTN_SUCCESS) {
        begin_run(ix->c);
        r = index_build(ix, n_seqs, max_distance, true);
        end_run(ix->c);
    }
    if (r != XTN_SUCCESS) {
        index_free(ix);
        return r;
    }
    *out = ix;
    return XTN_SUCCESS;
}

void xtn_index_destroy(xtn_index* ix) { index_free(ix); }

int xtn_index_stats(const xtn_index* ix, xtn_index_info* out) {
    if (!ix || !out) return XTN_ERR_ARG;
    out->n_seqs = ix->n;
    out->max_distance = ix->dmax;
    out->directory_bits = ix->dir_bits;
    out->n_records = (int64_t)ix->V;
    out->bytes = (int64_t)(ix->chars.cap + ix->offs.cap + ix->recs.cap + ix->dir.cap);
    out->ms_build = ix->ms_build;
    return XTN_SUCCESS;
}

xtn_context* xtn_index_context(xtn_index* ix) { return ix ? ix->c : nullptr; }

int xtn_index_query_device(xtn_index* ix, const xtn_args* args, const char* d_seqs, const uint32_t* d_offsets,
                           int32_t n_queries, int64_t* n_out) {
    if (!ix || !d_seqs || !d_offsets || n_queries < 1) {
        set_err("invalid arguments");
        return XTN_ERR_ARG;
    }
    XTN_TRY(check_args(args));
    XTN_CK(cudaSetDevice(ix->c->device));
    begin_run(ix->c);
    int r = index_query(ix, ix->c, ix->qb, reinterpret_cast<const uint8_t*>(d_seqs), d_offsets, n_queries,
                        args->distance, args->measure, true);
    end_run(ix->c);
    if (r == XTN_SUCCESS && n_out) *n_out = ix->c->n_out;
    return r;
}

int xtn_index_query(xtn_index* ix, const xtn_args* args, const char* seqs, const uint32_t* offsets, int32_t n_queries,
                    xtn_callback cb, void* user) {
    if (!ix || !seqs || !offsets || n_queries < 1) {
        set_err("invalid arguments");
        return XTN_ERR_ARG;
    }
    XTN_TRY(check_args(args));
    XTN_TRY(check_offsets(offsets, n_queries));
    xtn_context* c = ix->c;
    XTN_CK(cudaSetDevice(c->device));
    XTN_TRY(upload(c, seqs, offsets, n_queries));
    begin_run(c);
    int r = index_query(ix, c, ix->qb, P<uint8_t>(c->chars), P<uint32_t>(c->offs), n_queries, args->distance,
                        args->measure, false);
    end_run(c);
    if (r != XTN_SUCCESS) return r;
    return deliver(c, cb, user);
}

int xtn_index_serve(xtn_index* ix, const xtn_request* reqs, int32_t n_reqs, const xtn_serve_options* opt,
                    xtn_request_result* results, xtn_request_callback cb, void* user) {
    if (!ix || (!reqs && n_reqs > 0) || n_reqs < 0 || !results) {
        set_err("invalid arguments");
        return XTN_ERR_ARG;
    }
    for (int i = 0; i < n_reqs; i++) {
        const xtn_request& q = reqs[i];
        if (!q.seqs || !q.offsets || q.n_seqs < 1 || q.distance < 1 || q.distance > ix->dmax ||
            (q.measure != XTN_LEVENSHTEIN && q.measure != XTN_HAMMING)) {
            set_err("invalid request " + std::to_string(i));
            return XTN_ERR_ARG;
        }
        XTN_TRY(check_offsets(q.offsets, q.n_seqs));
        results[i] = xtn_request_result{-1.0, -1.0, 0, -1, XTN_ERROR};
    }
    const int64_t max_batch = opt && opt->max_batch_seqs > 0 ? opt->max_batch_seqs : (int64_t)1 << 20;
    const double frac = opt && opt->hbm_fraction > 0 && opt->hbm_fraction <= 1 ? opt->hbm_fraction : 0.5;
    const bool realtime = !opt || opt->realtime;
    const int nslots = opt && opt->slots > 0 ? std::min(opt->slots, kMaxServeSlots) : 2;
    const int device = ix->c->device;
    XTN_CK(cudaSetDevice(device));
    // slot 0 is the index's own context; the others get a context (stream, scratch) each
    struct Slot {
        xtn_context* c = nullptr;
        xtn_query_bufs own;
        xtn_query_bufs* qb = nullptr;
    };
    std::vector<Slot> slots(nslots);
    slots[0].c = ix->c;
    slots[0].qb = &ix->qb;
    auto free_slots = [&]() {
        for (int k = 1; k < nslots; k++) {
            if (!slots[k].c) continue;
            cudaStreamSynchronize(slots[k].c->stream);
            DevBuf* b[] = {&slots[k].own.qh, &slots[k].own.qrow, &slots[k].own.qlb, &slots[k].own.qcnt,
                           &slots[k].own.qcoff};
            for (DevBuf* x : b) release(*x);
            xtn_context_destroy(slots[k].c);
            slots[k].c = nullptr;
        }
    };
    for (int k = 1; k < nslots; k++) {
        const int r = xtn_context_create(device, &slots[k].c);
        if (r != XTN_SUCCESS) {
            free_slots();
            return r;
        }
        slots[k].qb = &slots[k].own;
    }
    // device memory for the largest batch a slot can form, reserved before the clock starts; the
    // memory budget is split over the slots and read once (a device-memory query can take tens
    // of milliseconds, far longer than a small batch)
    int64_t cap_by_d[3] = {0, 0, 0};
    {
        int64_t big = 0, big_chars = 0;
        int dbig = 1;
        for (int i = 0; i < n_reqs; i++) {
            big = std::max<int64_t>(big, reqs[i].n_seqs);
            big_chars = std::max<int64_t>(big_chars, reqs[i].offsets[reqs[i].n_seqs] - reqs[i].offsets[0]);
            dbig = std::max(dbig, reqs[i].distance);
        }
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        const double per_slot = (double)free_b * frac / nslots;
        const int64_t cap0 =
            std::max<int64_t>(1, std::min<int64_t>(max_batch, (int64_t)(per_slot / (double)query_bytes_per_seq(dbig))));
        const int64_t nres = std::min(std::max<int64_t>(big, std::min<int64_t>(cap0, 1 << 16)), cap0);
        for (int k = 0; k < nslots; k++) {
            const int r = index_reserve(slots[k].c, *slots[k].qb, nres, std::max<int64_t>(big_chars, nres * 24), dbig);
            if (r != XTN_SUCCESS) {
                free_slots();
                return r;
            }
        }
        for (int dd = 1; dd <= 2; dd++)
            cap_by_d[dd] = std::max<int64_t>(
                1, std::min<int64_t>(max_batch, (int64_t)(per_slot / (double)query_bytes_per_seq(dd))));
    }
    // requests in arrival order; a free slot takes the oldest ready request and the ready ones
    // of the same (distance, measure) that fit its budget, so a request that arrives while
    // another slot is busy with a large batch starts at once
    std::vector<int> order(n_reqs);
    for (int i = 0; i < n_reqs; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return reqs[a].arrival_s < reqs[b].arrival_s; });
    std::mutex mu, cb_mu;
    std::condition_variable cv;
    size_t next = 0;
    std::vector<int> ready;
    int batch_counter = 0, first_status = XTN_SUCCESS;
    std::string first_error;
    const double t0 = now_s();
    auto worker = [&](int k) {
        Slot& sl = slots[k];
        xtn_context* c = sl.c;
        if (cudaSetDevice(device) != cudaSuccess) return;
        std::vector<char> hchars;
        std::vector<uint32_t> hoffs;
        std::vector<xtn_int2> hp;
        std::vector<int8_t> hd;
        for (;;) {
            std::vector<int> batch;
            int d = 1, m = 0, batch_id = 0;
            int64_t cap = 1;
            {
                std::unique_lock<std::mutex> lk(mu);
                for (;;) {
                    if (first_status != XTN_SUCCESS) return;
                    const double now = now_s() - t0;
                    while (next < order.size() && (!realtime || reqs[order[next]].arrival_s <= now))
                        ready.push_back(order[next++]);
                    if (!ready.empty()) break;
                    if (next >= order.size()) return;  // every request admitted
                    const double wait = reqs[order[next]].arrival_s - now;
                    cv.wait_for(lk, std::chrono::duration<double>(std::max(wait, 0.0)));
                }
                d = reqs[ready[0]].distance;
                m = reqs[ready[0]].measure;
                cap = cap_by_d[d];
                std::vector<int> rest;
                int64_t seqs = 0;
                for (int r : ready) {
                    const xtn_request& q = reqs[r];
                    if (q.distance == d && q.measure == m && (batch.empty() || seqs + q.n_seqs <= cap)) {
                        batch.push_back(r);
                        seqs += q.n_seqs;
                    } else {
                        rest.push_back(r);
                    }
                }
                ready.swap(rest);
                batch_id = batch_counter++;
            }
            cv.notify_all();
            const double admitted = now_s() - t0;
            // a request larger than the budget runs in pieces of at most `cap` sequences
            struct Piece {
                int req, first, count;
                int64_t row0;
            };
            std::vector<Piece> pieces;
            for (int r : batch)
                for (int f = 0; f < reqs[r].n_seqs; f += (int)cap)
                    pieces.push_back(Piece{r, f, (int)std::min<int64_t>(cap, reqs[r].n_seqs - f), 0});
            std::vector<std::vector<xtn_int2>> rp(batch.size());
            std::vector<std::vector<int8_t>> rd(batch.size());
            std::vector<int> slot_of(n_reqs, -1);
            for (size_t q = 0; q < batch.size(); q++) slot_of[batch[q]] = (int)q;
            int status = XTN_SUCCESS;
            for (size_t p0 = 0; p0 < pieces.size() && status == XTN_SUCCESS;) {
                // pieces p0..p1 form one device round of at most `cap` sequences
                size_t p1 = p0;
                int64_t rows = 0;
                hchars.clear();
                hoffs.assign(1, 0);
                while (p1 < pieces.size() && (p1 == p0 || rows + pieces[p1].count <= cap)) {
                    Piece& pc = pieces[p1];
                    pc.row0 = rows;
                    const xtn_request& q = reqs[pc.req];
                    const uint32_t a0 = q.offsets[pc.first], base = hoffs.back();
                    hchars.insert(hchars.end(), q.seqs + a0, q.seqs + q.offsets[pc.first + pc.count]);
                    for (int i = 1; i <= pc.count; i++) hoffs.push_back(base + (q.offsets[pc.first + i] - a0));
                    rows += pc.count;
                    p1++;
                }
                status = upload(c, hchars.data(), hoffs.data(), (int)rows);
                if (status == XTN_SUCCESS) {
                    begin_run(c);
                    status = index_query(ix, c, *sl.qb, P<uint8_t>(c->chars), P<uint32_t>(c->offs), (int)rows, d, m,
                                         false);
                    end_run(c);
                }
                if (status != XTN_SUCCESS) break;
                const int64_t nout = c->n_out;
                hp.resize((size_t)nout);
                hd.resize((size_t)nout);
                if (nout > 0 &&
                    (cudaMemcpyAsync(hp.data(), c->out_pairs.p, sizeof(xtn_int2) * nout, cudaMemcpyDeviceToHost,
                                     c->stream) != cudaSuccess ||
                     cudaMemcpyAsync(hd.data(), c->out_dist.p, (size_t)nout, cudaMemcpyDeviceToHost, c->stream) !=
                         cudaSuccess ||
                     cudaStreamSynchronize(c->stream) != cudaSuccess)) {
                    set_err("copy of a batch result failed");
                    status = XTN_ERR_CUDA;
                    break;
                }
                // split by request: rows [row0, row0 + count) of the round belong to piece k
                std::vector<int64_t> starts;
                for (size_t k2 = p0; k2 < p1; k2++) starts.push_back(pieces[k2].row0);
                for (int64_t i = 0; i < nout; i++) {
                    const int64_t row = hp[i].y - ix->n;
                    const size_t k2 = p0 + (size_t)(std::upper_bound(starts.begin(), starts.end(), row) - starts.begin()) - 1;
                    const Piece& pc = pieces[k2];
                    const int sq = slot_of[pc.req];
                    rp[sq].push_back(xtn_int2{hp[i].x, (int32_t)(ix->n + pc.first + (row - pc.row0))});
                    rd[sq].push_back(hd[i]);
                }
                p0 = p1;
            }
            std::lock_guard<std::mutex> lk(cb_mu);  // callbacks come one at a time
            for (size_t q = 0; q < batch.size(); q++) {
                const int r = batch[q];
                xtn_request_result& res = results[r];
                res.admitted_s = admitted;
                res.batch = batch_id;
                res.status = status;
                if (status == XTN_SUCCESS) {
                    // a request split into pieces collects its pairs piece by piece: restore (x, y) order
                    std::vector<xtn_int2>& P2 = rp[q];
                    std::vector<int8_t>& D2 = rd[q];
                    bool sorted = true;
                    for (size_t i = 1; i < P2.size() && sorted; i++)
                        sorted = P2[i - 1].x < P2[i].x || (P2[i - 1].x == P2[i].x && P2[i - 1].y < P2[i].y);
                    if (!sorted) {
                        std::vector<size_t> idx(P2.size());
                        for (size_t i = 0; i < idx.size(); i++) idx[i] = i;
                        std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
                            return P2[a].x < P2[b].x || (P2[a].x == P2[b].x && P2[a].y < P2[b].y);
                        });
                        std::vector<xtn_int2> p3(P2.size());
                        std::vector<int8_t> d3(D2.size());
                        for (size_t i = 0; i < idx.size(); i++) {
                            p3[i] = P2[idx[i]];
                            d3[i] = D2[idx[i]];
                        }
                        P2.swap(p3);
                        D2.swap(d3);
                    }
                    res.n_out = (int64_t)P2.size();
                    if (cb) {
                        xtn_output o{P2.data(), D2.data(), nullptr, (int64_t)P2.size()};
                        cb(r, &o, user);
                    }
                }
                res.done_s = now_s() - t0;
            }
            if (status != XTN_SUCCESS) {
                std::lock_guard<std::mutex> lk2(mu);
                if (first_status == XTN_SUCCESS) {
                    first_status = status;
                    first_error = xtn_last_error();
                }
                cv.notify_all();
                return;
            }
        }
    };
    std::vector<std::thread> th;
    for (int k = 1; k < nslots; k++) th.emplace_back(worker, k);
    worker(0);
    for (auto& t : th) t.join();
    free_slots();
    if (first_status != XTN_SUCCESS) {
        set_err(first_error);
        return first_status;
    }
    return XTN_SUCCESS;
}

}  // extern "C"
