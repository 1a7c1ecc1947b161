// Stable LSD radix sort of (key, uint32 value) pairs with one "onesweep" kernel per 8-bit digit.
//
// Replaces cub::DeviceRadixSort::SortPairs as smallgwn calls it for Morton codes
// (detail/gwn_bvh_build_common.cuh:332-347): identical output for identical input, because both
// are stable sorts over key bits [0, key_bits).
//
// Per pass: every CTA claims a tile id from an atomic counter (so a tile only ever waits on tiles
// claimed before it), ranks its keys stably per warp with ballot-based digit matching, publishes
// its per-digit counts and resolves its global per-digit offsets by decoupled look-back, reading
// four predecessor tiles' words per round trip. The look-back spin is bounded; a timeout sets an
// error bit instead of hanging. Keys are staged in shared memory in digit order so global stores
// are coalesced runs.
#include "gwnb_internal.cuh"

#include <algorithm>

namespace gwnb {
namespace {

constexpr int k_threads = 256;
constexpr int k_warps = k_threads / 32;
constexpr std::uint32_t k_flag_agg = 1u << 30;
constexpr std::uint32_t k_flag_incl = 2u << 30;
constexpr std::uint32_t k_value_mask = (1u << 30) - 1u;

template <class K> struct sort_items;
// 12 / 8 keys per thread with three 256-thread blocks per SM (at most 85 registers): twice the
// resident tiles of 16 / 12 keys at two blocks, for 20 % less time per pass on 10M 32-bit keys
template <> struct sort_items<std::uint32_t> { static constexpr int value = 12; };
template <> struct sort_items<std::uint64_t> { static constexpr int value = 8; };
static_assert(k_threads * sort_items<std::uint32_t>::value == k_sort_tile_u32, "32-bit sort tile size");

__device__ inline std::uint32_t digit_of(std::uint32_t k, int shift, std::uint32_t mask) {
    return (k >> shift) & mask;
}
__device__ inline std::uint32_t digit_of(std::uint64_t k, int shift, std::uint32_t mask) {
    return static_cast<std::uint32_t>(k >> shift) & mask;
}

// Exclusive scan of one value per thread across a 256-thread block. `scratch` holds 8 words.
__device__ inline std::uint32_t block_exclusive_scan_256(std::uint32_t v, std::uint32_t *scratch,
                                                         std::uint32_t *total) {
    unsigned const lane = threadIdx.x & 31u;
    unsigned const warp = threadIdx.x >> 5;
    std::uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        std::uint32_t const t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= static_cast<unsigned>(o))
            incl += t;
    }
    if (lane == 31)
        scratch[warp] = incl;
    __syncthreads();
    std::uint32_t warp_prefix = 0, sum = 0;
#pragma unroll
    for (int w = 0; w < k_warps; ++w) {
        std::uint32_t const s = scratch[w];
        if (static_cast<unsigned>(w) < warp)
            warp_prefix += s;
        sum += s;
    }
    __syncthreads();
    if (total != nullptr)
        *total = sum;
    return warp_prefix + incl - v;
}

template <class K>
__global__ void __launch_bounds__(k_threads)
    k_sort_histogram(K const *__restrict__ keys, std::uint64_t n, int passes, int key_bits,
                     std::uint32_t *__restrict__ hist) {
    __shared__ std::uint32_t sh[8 * 256];
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x)
        sh[i] = 0;
    __syncthreads();
    for (std::uint64_t idx = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
         idx < n; idx += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        K const k = keys[idx];
        for (int p = 0; p < passes; ++p) {
            int const bits = min(8, key_bits - 8 * p);
            std::uint32_t const mask = (1u << bits) - 1u;
            atomicAdd(&sh[p * 256 + digit_of(k, 8 * p, mask)], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x)
        if (sh[i] != 0)
            atomicAdd(&hist[i], sh[i]);
}

template <class K, int Items>
__global__ void __launch_bounds__(k_threads, 3)
    k_onesweep(K const *__restrict__ keys_in, std::uint32_t const *__restrict__ vals_in,
               K *__restrict__ keys_out, std::uint32_t *__restrict__ vals_out, std::uint64_t n,
               int shift, std::uint32_t mask, std::uint32_t const *__restrict__ hist,
               std::uint32_t *tile_status, std::uint32_t *tile_counter, unsigned int *status, long long wait_limit) {
    constexpr int k_tile = k_threads * Items;
    __shared__ std::uint32_t s_warp_hist[k_warps][256];
    __shared__ std::uint32_t s_block_excl[256];
    __shared__ std::uint32_t s_global_base[256];
    __shared__ std::uint32_t s_scan[k_warps];
    __shared__ std::uint32_t s_tile;
    __shared__ K s_keys[k_tile];
    __shared__ std::uint32_t s_vals[k_tile];

    unsigned const tid = threadIdx.x;
    unsigned const lane = tid & 31u;
    unsigned const warp = tid >> 5;
    if (tid == 0)
        s_tile = atomicAdd(tile_counter, 1u);
    for (int i = tid; i < k_warps * 256; i += k_threads)
        (&s_warp_hist[0][0])[i] = 0;
    __syncthreads();
    std::uint32_t const tile = s_tile;
    std::uint64_t const tile_base = static_cast<std::uint64_t>(tile) * k_tile;

    K key[Items];
    std::uint32_t val[Items];
    std::uint32_t dig[Items];
    std::uint32_t rank[Items];
#pragma unroll
    for (int r = 0; r < Items; ++r) {
        std::uint64_t const idx = tile_base + warp * (32u * Items) + r * 32u + lane;
        bool const valid = idx < n;
        key[r] = valid ? keys_in[idx] : K(0);
        val[r] = valid ? (vals_in != nullptr ? vals_in[idx] : static_cast<std::uint32_t>(idx)) : 0u;
        dig[r] = valid ? digit_of(key[r], shift, mask) : 256u;
    }

    // Warp-level stable ranking: rounds in index order, lanes in index order within a round.
    unsigned const lt_mask = (1u << lane) - 1u;
    std::uint32_t *const wh = s_warp_hist[warp];
#pragma unroll
    for (int r = 0; r < Items; ++r) {
        std::uint32_t const d = dig[r];
        bool const valid = d < 256u;
        unsigned peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            bool const bit = ((d >> b) & 1u) != 0u;
            unsigned const bb = __ballot_sync(0xffffffffu, bit);
            peers &= bit ? bb : ~bb;
        }
        std::uint32_t base = 0;
        if (valid)
            base = wh[d];
        __syncwarp();
        if (valid) {
            rank[r] = base + __popc(peers & lt_mask);
            if ((__ffs(peers) - 1) == static_cast<int>(lane))
                wh[d] = base + __popc(peers);
        }
        __syncwarp();
    }
    __syncthreads();

    // Per digit: exclusive offsets of each warp and the tile's count.
    std::uint32_t count = 0;
    {
        std::uint32_t const d = tid;
#pragma unroll
        for (int w = 0; w < k_warps; ++w) {
            std::uint32_t const t = s_warp_hist[w][d];
            s_warp_hist[w][d] = count;
            count += t;
        }
    }
    std::uint32_t const block_excl = block_exclusive_scan_256(count, s_scan, nullptr);
    std::uint32_t const hist_excl = block_exclusive_scan_256(hist[tid], s_scan, nullptr);
    s_block_excl[tid] = block_excl;

    // Decoupled look-back for this digit across earlier tiles.
    {
        std::uint32_t const d = tid;
        std::uint32_t excl = 0;
        if (tile == 0) {
            atomicExch(&tile_status[d], k_flag_incl | count);
        } else {
            atomicExch(&tile_status[static_cast<std::size_t>(tile) * 256 + d], k_flag_agg | count);
            long long spins = 0;
            std::int64_t j = static_cast<std::int64_t>(tile) - 1;
            // 4 predecessors per round trip: their words are read together, then consumed in
            // order until an unpublished one (re-read from there) or an inclusive prefix
            bool done = false;
            while (!done && j >= 0) {
                std::uint32_t w[4];
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    w[k] = j - k >= 0 ? *reinterpret_cast<volatile std::uint32_t *>(&tile_status[(j - k) * 256 + d])
                                      : 0u;
                int consumed = 0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (done || consumed != k)
                        continue;
                    if (j - k < 0) {
                        done = true;
                        continue;
                    }
                    std::uint32_t const f = w[k] & ~k_value_mask;
                    if (f == 0u)
                        continue;
                    excl += w[k] & k_value_mask;
                    ++consumed;
                    if (f == k_flag_incl)
                        done = true;
                }
                j -= consumed;
                if (!done && consumed == 0 && ++spins > wait_limit) {
                    atomicOr(status, k_err_wait_timeout);
                    break;
                }
            }
            atomicExch(&tile_status[static_cast<std::size_t>(tile) * 256 + d],
                       k_flag_incl | ((excl + count) & k_value_mask));
        }
        s_global_base[d] = hist_excl + excl;
    }
    __syncthreads();

#pragma unroll
    for (int r = 0; r < Items; ++r) {
        std::uint32_t const d = dig[r];
        if (d < 256u) {
            std::uint32_t const pos = s_block_excl[d] + s_warp_hist[warp][d] + rank[r];
            s_keys[pos] = key[r];
            s_vals[pos] = val[r];
        }
    }
    __syncthreads();

    std::uint64_t const remaining = n - tile_base;
    std::uint32_t const tile_n =
        remaining < static_cast<std::uint64_t>(k_tile) ? static_cast<std::uint32_t>(remaining)
                                                       : static_cast<std::uint32_t>(k_tile);
    for (std::uint32_t i = tid; i < tile_n; i += k_threads) {
        K const k = s_keys[i];
        std::uint32_t const d = digit_of(k, shift, mask);
        std::uint64_t const dest =
            static_cast<std::uint64_t>(s_global_base[d]) + (i - s_block_excl[d]);
        keys_out[dest] = k;
        vals_out[dest] = s_vals[i];
    }
}

template <class K>
int sort_impl(K const *keys_in, K *keys_out, std::uint32_t const *vals_in,
              std::uint32_t *vals_out, std::uint64_t n, int key_bits, cudaStream_t s,
              unsigned int *status) {
    constexpr int k_items = sort_items<K>::value;
    constexpr std::uint64_t k_tile = static_cast<std::uint64_t>(k_threads) * k_items;
    if (n == 0)
        return GWNB_OK;
    if (n >= (std::uint64_t(1) << 30))
        return set_error(GWNB_INVALID_ARGUMENT, "radix sort: at most 2^30 - 1 elements per call.");
    if (key_bits <= 0 || key_bits > static_cast<int>(sizeof(K) * 8))
        return set_error(GWNB_INVALID_ARGUMENT, "radix sort: key_bits out of range.");
    int const passes = (key_bits + 7) / 8;
    std::uint64_t const tiles = (n + k_tile - 1) / k_tile;

    K *keys_tmp = nullptr;
    std::uint32_t *vals_tmp = nullptr;
    std::uint32_t *words = nullptr; // hist (passes*256) | counters (passes) | status (passes*tiles*256)
    std::size_t const word_count = passes * 256 + passes + passes * tiles * 256;
    scratch_guard guard(s);
    guard.hold(keys_tmp, vals_tmp, words);
    GWNB_TRY(alloc(&keys_tmp, n, s));
    GWNB_TRY(alloc(&vals_tmp, n, s));
    GWNB_TRY(alloc(&words, word_count, s));
    GWNB_CUDA_TRY(cudaMemsetAsync(words, 0, word_count * sizeof(std::uint32_t), s));
    std::uint32_t *hist = words;
    std::uint32_t *counters = words + passes * 256;
    std::uint32_t *tile_status = counters + passes;

    int const sms = device_sm_count();
    unsigned const hist_grid = static_cast<unsigned>(
        std::min<std::uint64_t>((n + k_threads - 1) / k_threads, static_cast<std::uint64_t>(sms) * 8));
    note_launch(), k_sort_histogram<K><<<hist_grid, k_threads, 0, s>>>(keys_in, n, passes, key_bits, hist);

    // Ping-pong so that the last pass lands in the output buffers.
    long long const limit = wait_limit();
    bool to_out = (passes % 2) == 1;
    K const *src_k = keys_in;
    std::uint32_t const *src_v = vals_in;
    for (int p = 0; p < passes; ++p) {
        K *dst_k = to_out ? keys_out : keys_tmp;
        std::uint32_t *dst_v = to_out ? vals_out : vals_tmp;
        int const bits = std::min(8, key_bits - 8 * p);
        std::uint32_t const mask = (1u << bits) - 1u;
        note_launch(), k_onesweep<K, k_items><<<static_cast<unsigned>(tiles), k_threads, 0, s>>>(
            src_k, src_v, dst_k, dst_v, n, 8 * p, mask, hist + p * 256,
            tile_status + static_cast<std::size_t>(p) * tiles * 256, counters + p, status, limit);
        src_k = dst_k;
        src_v = dst_v;
        to_out = !to_out;
    }
    GWNB_CUDA_TRY(cudaGetLastError());
    release(keys_tmp, s);
    release(vals_tmp, s);
    release(words, s);
    return GWNB_OK;
}

// The same passes as sort_impl over caller-provided scratch: keys_tmp (n keys), vals_tmp (n
// words) and `words` (histograms, tile counters, tile status), which is cleared here.
template <class K>
int sort_in_scratch(K const *keys_in, K *keys_out, std::uint32_t const *vals_in, std::uint32_t *vals_out,
                    std::uint64_t n, int key_bits, K *keys_tmp, std::uint32_t *vals_tmp, std::uint32_t *words,
                    cudaStream_t s, unsigned int *status) {
    constexpr int k_items = sort_items<K>::value;
    constexpr std::uint64_t k_tile = static_cast<std::uint64_t>(k_threads) * k_items;
    if (n == 0)
        return GWNB_OK;
    int const passes = (key_bits + 7) / 8;
    std::uint64_t const tiles = (n + k_tile - 1) / k_tile;
    std::size_t const word_count = passes * 256 + passes + passes * tiles * 256;
    GWNB_CUDA_TRY(cudaMemsetAsync(words, 0, word_count * sizeof(std::uint32_t), s));
    std::uint32_t *hist = words;
    std::uint32_t *counters = words + passes * 256;
    std::uint32_t *tile_status = counters + passes;
    int const sms = device_sm_count();
    unsigned const hist_grid = static_cast<unsigned>(
        std::min<std::uint64_t>((n + k_threads - 1) / k_threads, static_cast<std::uint64_t>(sms) * 8));
    note_launch(), k_sort_histogram<K><<<hist_grid, k_threads, 0, s>>>(keys_in, n, passes, key_bits, hist);
    long long const limit = wait_limit();
    bool to_out = (passes % 2) == 1;
    K const *src_k = keys_in;
    std::uint32_t const *src_v = vals_in;
    for (int p = 0; p < passes; ++p) {
        K *dst_k = to_out ? keys_out : keys_tmp;
        std::uint32_t *dst_v = to_out ? vals_out : vals_tmp;
        int const bits = std::min(8, key_bits - 8 * p);
        std::uint32_t const mask = (1u << bits) - 1u;
        note_launch(), k_onesweep<K, k_items><<<static_cast<unsigned>(tiles), k_threads, 0, s>>>(
            src_k, src_v, dst_k, dst_v, n, 8 * p, mask, hist + p * 256,
            tile_status + static_cast<std::size_t>(p) * tiles * 256, counters + p, status, limit);
        src_k = dst_k;
        src_v = dst_v;
        to_out = !to_out;
    }
    GWNB_CUDA_TRY(cudaGetLastError());
    return GWNB_OK;
}

} // namespace

// One real onesweep pass whose first tile is never processed: two tiles of keys, the tile counter
// starting at 1 and one block, so the block takes tile 1 and its look-back waits on tile 0, which
// nothing publishes. The wait gives up after wait_limit() polls and sets k_err_wait_timeout in
// *status; every access stays inside the two-tile buffers (tile 1's prefix is then what it gathered
// before giving up, zero, and its keys land in the first tile's positions).
int onesweep_wait_probe(unsigned int *status, cudaStream_t s) {
    constexpr int k_items = sort_items<std::uint32_t>::value;
    constexpr std::uint64_t k_tile = static_cast<std::uint64_t>(k_threads) * k_items;
    constexpr std::uint64_t n = 2 * k_tile;
    std::uint32_t *keys = nullptr, *out_keys = nullptr, *out_vals = nullptr, *words = nullptr;
    // words: histogram (256) | tile counter (1) | tile status (2 tiles x 256)
    std::size_t const word_count = 256 + 1 + 2 * 256;
    scratch_guard guard(s);
    guard.hold(keys, out_keys, out_vals, words);
    GWNB_TRY(alloc(&keys, n, s));
    GWNB_TRY(alloc(&out_keys, n, s));
    GWNB_TRY(alloc(&out_vals, n, s));
    GWNB_TRY(alloc(&words, word_count, s));
    GWNB_CUDA_TRY(cudaMemsetAsync(keys, 0, n * sizeof(std::uint32_t), s));
    GWNB_CUDA_TRY(cudaMemsetAsync(words, 0, word_count * sizeof(std::uint32_t), s));
    std::uint32_t const first_tile = 1;
    GWNB_CUDA_TRY(cudaMemcpyAsync(words + 256, &first_tile, sizeof(first_tile), cudaMemcpyHostToDevice, s));
    note_launch(), k_sort_histogram<std::uint32_t><<<2, k_threads, 0, s>>>(keys, n, 1, 8, words);
    note_launch(), k_onesweep<std::uint32_t, k_items><<<1, k_threads, 0, s>>>(
        keys, nullptr, out_keys, out_vals, n, 0, 0xffu, words, words + 257, words + 256, status, wait_limit());
    cudaError_t const e = cudaGetLastError();
    GWNB_CUDA_TRY(cudaStreamSynchronize(s));
    release(keys, s);
    release(out_keys, s);
    release(out_vals, s);
    release(words, s);
    if (e != cudaSuccess)
        return set_cuda_error(e, "onesweep wait probe");
    return GWNB_OK;
}

std::size_t radix_sort_u32_scratch_words(std::uint64_t n, int key_bits) {
    constexpr std::uint64_t k_tile = static_cast<std::uint64_t>(k_threads) * sort_items<std::uint32_t>::value;
    int const passes = (key_bits + 7) / 8;
    std::uint64_t const tiles = (n + k_tile - 1) / k_tile;
    return static_cast<std::size_t>(passes * 256 + passes + passes * tiles * 256);
}

int radix_sort_pairs_u32_in_scratch(std::uint32_t const *keys_in, std::uint32_t *keys_out,
                                    std::uint32_t const *values_in, std::uint32_t *values_out, std::uint64_t n,
                                    int key_bits, std::uint32_t *keys_tmp, std::uint32_t *vals_tmp,
                                    std::uint32_t *words, cudaStream_t s, unsigned int *status) {
    return sort_in_scratch<std::uint32_t>(keys_in, keys_out, values_in, values_out, n, key_bits, keys_tmp, vals_tmp,
                                          words, s, status);
}

int radix_sort_pairs(void const *keys_in, void *keys_out, std::uint32_t const *values_in,
                     std::uint32_t *values_out, std::uint64_t n, int key_bytes, int key_bits,
                     cudaStream_t s, unsigned int *status) {
    if (key_bytes == 4)
        return sort_impl<std::uint32_t>(static_cast<std::uint32_t const *>(keys_in),
                                        static_cast<std::uint32_t *>(keys_out), values_in,
                                        values_out, n, key_bits, s, status);
    if (key_bytes == 8)
        return sort_impl<std::uint64_t>(static_cast<std::uint64_t const *>(keys_in),
                                        static_cast<std::uint64_t *>(keys_out), values_in,
                                        values_out, n, key_bits, s, status);
    return set_error(GWNB_INVALID_ARGUMENT, "radix sort: key_bytes must be 4 or 8.");
}

} // namespace gwnb
