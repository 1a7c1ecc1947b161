// Taylor order and accuracy scale chosen from an error target (no smallgwn counterpart).
//
// smallgwn leaves the Taylor order (a template parameter) and the accuracy scale beta to the
// caller. Given a caller's error bound, this picks them on a sample of the caller's own queries:
// the sample's FP64 exact winding numbers are the reference (gwnb_winding_exact_geometry_fp64's
// kernel); for every order whose moments the caller supplies, the smallest candidate beta whose
// maximum error on the sample stays within the bound is that order's candidate (the error falls as
// beta grows, the cost rises); the candidates are timed on the sample with CUDA events and the
// fastest is chosen. The stack capacity is the tree's exact internal stack bound. Everything runs
// on the caller's stream; the call synchronizes it.
#include "gwnb_internal.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

namespace gwnb {

int exact_batch_f64(gwnb_geometry_f32 const &g, float const *qx, float const *qy, float const *qz, double *out,
                    std::uint64_t nq, cudaStream_t s);
int taylor_batch(taylor_request const &r, cudaStream_t s);

namespace {

// Maximum of |w - ref| over the sample as ordered bits of a non-negative float (NaN counts as +inf).
__global__ void __launch_bounds__(256)
    k_max_abs_error(float const *__restrict__ w, double const *__restrict__ ref, std::uint64_t n, unsigned int *out) {
    float e = 0.0f;
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        double const d = fabs(static_cast<double>(w[i]) - ref[i]);
        float const f = d == d ? static_cast<float>(d) : __int_as_float(0x7f800000);
        e = fmaxf(e, f);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        e = fmaxf(e, __shfl_xor_sync(0xffffffffu, e, o));
    if ((threadIdx.x & 31u) == 0u)
        atomicMax(out, __float_as_uint(e));
}

} // namespace
} // namespace gwnb

using namespace gwnb;

extern "C" {

int gwnb_taylor_select_f32(const gwnb_geometry_f32 *geometry, const gwnb_bvh4_f32 *bvh_in,
                           const gwnb_moment4_f32 *const *moments, const float *qx, const float *qy, const float *qz,
                           uint64_t n, float max_error, const float *betas, int beta_count, int near_precision,
                           gwnb_taylor_choice *out, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::taylor_select");
    if (out == nullptr || moments == nullptr || betas == nullptr || beta_count <= 0)
        return set_error(GWNB_INVALID_ARGUMENT, "taylor select: null argument or no candidate accuracy scale.");
    if (!geometry_valid(geometry) || !bvh_valid(bvh_in) || geometry->triangle_count != bvh_in->primitive_count)
        return set_error(GWNB_INVALID_ARGUMENT, "taylor select: geometry and BVH must be valid and match.");
    if (!(max_error > 0.0f))
        return set_error(GWNB_INVALID_ARGUMENT, "taylor select: the error bound must be positive.");
    if (n == 0 || !has_storage(qx, n) || !has_storage(qy, n) || !has_storage(qz, n))
        return set_error(GWNB_INVALID_ARGUMENT, "taylor select: the query sample must be non-empty device storage.");
    if (n > 0xffffffffull)
        return set_error(GWNB_INVALID_ARGUMENT, "taylor select: the sample exceeds 2^32 - 1 queries.");
    if (near_precision != GWNB_NEAR_PLAIN && near_precision != GWNB_NEAR_COMPENSATED)
        return set_error(GWNB_INVALID_ARGUMENT, "Unknown near-field precision mode.");
    for (int i = 0; i < beta_count; ++i)
        if (!(betas[i] >= 0.0f))
            return set_error(GWNB_INVALID_ARGUMENT, "Taylor accuracy scale must be nonnegative.");
    bool any = false;
    for (int o = 0; o < 3; ++o)
        if (moments[o] != nullptr) {
            if (moments[o]->order != o || !moment_valid_for(moments[o], bvh_in))
                return set_error(GWNB_INVALID_ARGUMENT, "taylor select: moments[order] must be valid for the BVH.");
            any = true;
        }
    if (!any)
        return set_error(GWNB_INVALID_ARGUMENT, "taylor select: no moments given.");
    if (ref_internal(bvh_in->root.reference) && bvh_in->internal_stack_bound > 128)
        return set_error(GWNB_INVALID_ARGUMENT, "Traversal stack bounds above 128 are not supported.");

    cudaStream_t const s = as_cuda(stream);
    auto *b = const_cast<gwnb_bvh4_f32 *>(bvh_in);
    GWNB_TRY(ensure_bvh_aux(b, s));
    auto *a = reinterpret_cast<bvh_aux_impl *>(b->aux);
    std::vector<float> sorted(betas, betas + beta_count);
    std::sort(sorted.begin(), sorted.end());

    double *ref = nullptr;
    float *w = nullptr;
    unsigned int *err = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = GWNB_OK;
    auto cleanup = [&]() {
        release(ref, s);
        release(w, s);
        release(err, s);
        if (e0 != nullptr)
            cudaEventDestroy(e0);
        if (e1 != nullptr)
            cudaEventDestroy(e1);
    };
    if ((rc = alloc(&ref, n, s)) != GWNB_OK || (rc = alloc(&w, n, s)) != GWNB_OK || (rc = alloc(&err, 1, s)) != GWNB_OK) {
        cleanup();
        return rc;
    }
    if ((rc = exact_batch_f64(*geometry, qx, qy, qz, ref, n, s)) != GWNB_OK) {
        cleanup();
        return rc;
    }
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cleanup();
        return set_cuda_error(cudaGetLastError(), "taylor select events");
    }

    auto request = [&](int order, float beta) {
        auto const *ma = reinterpret_cast<moment_aux_impl *>(moments[order]->aux);
        taylor_request r{};
        r.order = order;
        r.qnodes = ma != nullptr ? ma->qnodes : nullptr;
        r.qcounts = ma != nullptr ? ma->qcounts : nullptr;
        r.tri48 = a->tri48;
        r.primitive_count = b->primitive_count;
        r.node_count = b->node_count;
        r.root_ref = b->root.reference;
        r.root_bounds = a->root_bounds;
        r.qx = qx;
        r.qy = qy;
        r.qz = qz;
        r.out = w;
        r.n = n;
        r.accuracy_scale = beta;
        r.block = 256;
        r.stack_capacity = std::max<int>(static_cast<int>(b->internal_stack_bound), 1);
        r.sort_queries = 1;
        r.near_mode = near_precision;
        r.fp64_threshold = 1.0f / 16.0f;
        r.fp64_count = a->fp64_count;
        r.status = a->status;
        return r;
    };
    auto sample_error = [&](int order, float beta, float *e) -> int {
        GWNB_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(unsigned int), s));
        GWNB_TRY(taylor_batch(request(order, beta), s));
        unsigned const grid = static_cast<unsigned>(std::min<std::uint64_t>((n + 255) / 256, 1024));
        note_launch(), k_max_abs_error<<<grid, 256, 0, s>>>(w, ref, n, err);
        GWNB_CUDA_TRY(cudaGetLastError());
        unsigned int bits = 0;
        GWNB_CUDA_TRY(cudaMemcpyAsync(&bits, err, sizeof(bits), cudaMemcpyDeviceToHost, s));
        GWNB_CUDA_TRY(cudaStreamSynchronize(s));
        std::memcpy(e, &bits, sizeof(bits));
        return GWNB_OK;
    };
    auto sample_ms = [&](int order, float beta, float *ms) -> int {
        GWNB_TRY(taylor_batch(request(order, beta), s)); // warm
        constexpr int reps = 3;
        GWNB_CUDA_TRY(cudaEventRecord(e0, s));
        for (int i = 0; i < reps; ++i)
            GWNB_TRY(taylor_batch(request(order, beta), s));
        GWNB_CUDA_TRY(cudaEventRecord(e1, s));
        GWNB_CUDA_TRY(cudaEventSynchronize(e1));
        GWNB_CUDA_TRY(cudaEventElapsedTime(ms, e0, e1));
        *ms /= reps;
        return GWNB_OK;
    };

    gwnb_taylor_choice best{};
    best.order = -1;
    int passing = 0;
    for (int o = 0; o < 3 && rc == GWNB_OK; ++o) {
        if (moments[o] == nullptr)
            continue;
        for (float beta : sorted) {
            float e = 0.0f;
            if ((rc = sample_error(o, beta, &e)) != GWNB_OK)
                break;
            if (!(e <= max_error))
                continue;
            float ms = 0.0f;
            if ((rc = sample_ms(o, beta, &ms)) != GWNB_OK)
                break;
            ++passing;
            if (best.order < 0 || ms < best.sample_ms)
                best = gwnb_taylor_choice{o, beta, e, ms, 0, 0};
            break; // larger scales of this order only cost more
        }
    }
    cleanup();
    if (rc != GWNB_OK)
        return rc;
    if (best.order < 0)
        return set_error(GWNB_INVALID_ARGUMENT, "taylor select: no candidate order and accuracy scale meets the bound "
                                                "on the sample.");
    best.stack_capacity = ref_internal(b->root.reference) ? static_cast<int>(b->internal_stack_bound) : 0;
    best.candidates_passing = passing;
    *out = best;
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

} // extern "C"
