// story.cu -- Starlab story-format snapshots read on the GPU: the dyn-class
// reader get_dyn (src/node/dyn/util/dyn_io.C:280-296 -> get_node,
// src/node/util/tree_io.C:253-410) as a data-parallel pass over the text.
//
// The reference reads a snapshot line by line with a recursive descent
// (one istream, one node at a time).  Here every line is handled by its
// own thread and the nesting is recovered from bracket depth:
//   1. newline index: per 16 KB tile the '\n' bytes are counted, the counts
//      scanned, and every newline's offset written in order;
//   2. one thread per line classifies it (util_io.C:94-136 rules: lines cut
//      at 254 characters; a line opens/closes a section when its first
//      character is '(' / ')', the next one naming it; otherwise
//      "keyword = value" or nothing);
//   3. bracket depth by a scan; the snapshot list ends at the first empty
//      line at depth 0 (check_and_skip_input_line, util_io.C:54-82);
//   4. each line's enclosing open line: chunks of 64 lines record the last
//      open line at every depth, a scan over chunks gives each chunk the
//      open lines around its start, and each chunk then walks its lines with
//      that stack;
//   5. context: an open line directly in a particle (or at the top) named
//      P, D, H, S or L is a section; any other open line -- and every open
//      line inside a Log, Dynamics, Hydro or Star section -- is a chapter,
//      transparent for the lines it holds (the reference reads Log chapters
//      by their raw first character with matching titles, story.C:172-203,
//      and treats lines inside D/H/S as content up to the first ")D", ")H",
//      ")S" line);
//   6. Particle sections are numbered by a scan (pre-order node ids), each
//      node's parent is its context, its subtree ends at its close line;
//   7. "m", "r", "v", "system_time" lines of a Dynamics section and "i",
//      "name" lines of a particle are claimed by the node, the last line of
//      each kind winning (atomicMax of the line number), and converted with
//      strtod / strtol semantics (story_num.h, bit-exact);
//   8. unless raw: check_and_correct_node (dyn_io.C:94-146), every parent's
//      mass := the sum of its daughters', daughters moved to their centre of
//      mass, level by level from the deepest, each parent's sums taken in
//      daughter order exactly as the reference adds them (no FMA);
//   9. leaves with positions and velocities relative to the root
//      (something_relative_to_root, dyn_tt.C:94-110).
// Inputs the two readings could read differently are rejected with the line
// number instead of being read differently: a section line indented by
// blanks, a chapter inside a Dynamics/Hydro/Star section named with that
// section's letter, mismatched closing lines, and forms story_num.h does not
// convert.
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>
#include "story_num.h"

// The library is built with hidden visibility; only the C ABI is exported.
#pragma GCC visibility push(default)
#include "../../include/g6b200_story.h"
#pragma GCC visibility pop

namespace storyk {

constexpr int kLineMax = 254;  // get_line keeps 254 characters (MAX_INPUT_LINE_LENGTH 255)
constexpr int kMaxDepth = 32;  // bracket nesting supported
constexpr int kChunk = 32;     // lines per thread in the enclosing-line pass
constexpr int kScanTile = 4096;
constexpr int kNlThreads = 256, kNlBytes = 64, kNlTile = kNlThreads * kNlBytes;

// Line tag: code | flags | kind/key << 8 | value offset << 16.
enum : uint32_t { C_OTHER = 0, C_OPEN = 1, C_CLOSE = 2, C_KEY = 3, C_INDENT = 4 };
enum : uint32_t { F_EMPTY = 8, F_LONG = 16, F_STRUCT = 32 };
enum : int { K_M = 1, K_R, K_V, K_TIME, K_RTIME, K_I, K_NAME, K_N, K_OTHER };  // keyword ids of key lines
enum : int { FLD_M = 0, FLD_R, FLD_V, FLD_TIME, FLD_I, FLD_NAME, FLD_COUNT };

// Error codes (low byte of the error word; the line number above it).
enum : int {
    E_NUL = 1, E_INDENT, E_TOP, E_CLOSE0, E_DEPTH, E_EOF, E_KIND, E_TITLE, E_CONFLICT, E_LONG, E_EMPTY,
    E_KEYWORD, E_VECTOR, E_NUMBER, E_SCAN
};
__host__ const char *error_text(int code) {
    switch (code) {
        case E_NUL: return "NUL byte in the text";
        case E_INDENT: return "section line indented by blanks (not supported)";
        case E_TOP: return "expected (Particle";
        case E_CLOSE0: return "closing line without an opening one";
        case E_DEPTH: return "sections nested deeper than 32";
        case E_EOF: return "end of text inside a Particle";
        case E_KIND: return "closing line does not match its opening line";
        case E_TITLE: return "story chapter closing title differs from its opening title";
        case E_CONFLICT: return "chapter inside a Dynamics/Hydro/Star section named like the section (not supported)";
        case E_LONG: return "story line too long";
        case E_EMPTY: return "empty line inside a story chapter";
        case E_KEYWORD: return "unexpected keyword in a Particle";
        case E_VECTOR: return "expected three reals";
        case E_NUMBER: return "number form not supported (hexadecimal, NaN payload or more than 40 digits)";
        case E_SCAN: return "internal: a device scan's wait for an earlier tile timed out";
        default: return "parse error";
    }
}

__device__ __forceinline__ void report(unsigned long long *err, long long line, int code) {
    atomicMin(err, ((unsigned long long)line << 8) | (unsigned long long)code);
}

__device__ __forceinline__ uint32_t code_of(uint32_t t) { return t & 7u; }
__device__ __forceinline__ int kind_of(uint32_t t) { return (int)((t >> 8) & 0xffu); }
__device__ __forceinline__ int voff_of(uint32_t t) { return (int)((t >> 16) & 0xffu); }
__device__ __forceinline__ int delta_of(uint32_t t) {
    const uint32_t c = code_of(t);
    return c == C_OPEN ? 1 : (c == C_CLOSE ? -1 : 0);
}

// Byte offsets are 64-bit (texts above 2 GB); line and node numbers 32-bit.
struct LineRange {
    const long long *nl;
    int nnl;
    long long len;
    __device__ __forceinline__ void get(int k, long long &s, long long &e) const {
        s = k == 0 ? 0 : nl[k - 1] + 1;
        e = k < nnl ? nl[k] : len;
    }
    // the line's first byte and its length after get_line's cut at 254
    __device__ __forceinline__ int span(int k, long long &s) const {
        long long e;
        get(k, s, e);
        return (int)min(e - s, (long long)kLineMax);
    }
};

// ---------------------------------------------------------------------------
// Block scans.

template <int NT, class T = int>
__device__ __forceinline__ T block_excl_sum(T v, T *total) {
    __shared__ T ws[NT / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        T s = lane < NT / 32 ? ws[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const T y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < NT / 32) ws[lane] = s;
    }
    __syncthreads();
    const T before = (w ? ws[w - 1] : 0) + x - v;
    if (total) *total = ws[NT / 32 - 1];
    __syncthreads();
    return before;
}

template <int NT>
__device__ __forceinline__ int block_excl_max(int v) {
    __shared__ int ws[NT / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x = max(x, y);
    }
    int ex = __shfl_up_sync(0xffffffffu, x, 1);
    if (lane == 0) ex = -1;
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = lane < NT / 32 ? ws[lane] : -1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s = max(s, y);
        }
        if (lane < NT / 32) ws[lane] = s;
    }
    __syncthreads();
    const int r = max(ex, w ? ws[w - 1] : -1);
    __syncthreads();
    return r;
}

// Exclusive sum of n values in one block (the newline index's block counts).
template <class T>
__global__ void __launch_bounds__(1024) scan_tiles_kernel(T *v, int n, T *total) {
    const int per = (n + 1023) / 1024;
    const int b = threadIdx.x * per, e = min(n, b + per);
    T s = 0;
    for (int k = b; k < e; ++k) s += v[k];
    T tot;
    T run = block_excl_sum<1024, T>(s, &tot);
    for (int k = b; k < e; ++k) {
        const T x = v[k];
        v[k] = run;
        run += x;
    }
    if (threadIdx.x == 0 && total) *total = tot;
}

// Single-pass exclusive sum (decoupled look-back): each CTA takes the next
// tile by ticket (so every tile it waits for belongs to a CTA already
// running), publishes its own sum, then walks back over the earlier tiles'
// published sums until one carries its inclusive prefix.  A status word is
// value | flag << 32 | epoch << 34; the epoch (one per scan) tells this
// scan's words from an earlier scan's.  Waits are bounded: after kScanWaitNs
// the scan reports E_SCAN and goes on.
constexpr unsigned long long kScanWaitNs = 1000000000ull;
enum : unsigned { SCAN_AGG = 1, SCAN_PREFIX = 2 };

__device__ __forceinline__ unsigned long long story_clock_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <class F>
__global__ void __launch_bounds__(256) scan1_kernel(F f, long long n, int *out, int *total,
                                                    unsigned long long *status, unsigned long long *ticket,
                                                    unsigned long long base, unsigned epoch, int ntiles,
                                                    unsigned long long *err) {
    __shared__ int s_tile, s_prefix;
    if (threadIdx.x == 0) s_tile = (int)(atomicAdd(ticket, 1ull) - base);
    __syncthreads();
    const int tile = s_tile;
    if (tile < 0 || tile >= ntiles) {  // tickets out of step with the host's count: report, write nothing
        if (threadIdx.x == 0) report(err, 0, E_SCAN);
        return;
    }
    // f is evaluated striped (element b + j * 256 + thread: coalesced), the
    // values pass through shared memory to this thread's 16 consecutive
    // elements (padded rows: one word per 32), and the results go back out
    // striped.
    __shared__ int sv[kScanTile + kScanTile / 32];
    const long long b = (long long)tile * kScanTile;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const int i = j * 256 + threadIdx.x;
        sv[i + i / 32] = b + i < n ? f(b + i) : 0;
    }
    __syncthreads();
    int v[16], sum = 0;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const int i = threadIdx.x * 16 + j;
        v[j] = sv[i + i / 32];
        sum += v[j];
    }
    int agg;
    const int excl = block_excl_sum<256>(sum, &agg);
    if (threadIdx.x == 0) {
        const unsigned long long ep = (unsigned long long)epoch << 34;
        int prefix = 0;
        if (tile > 0) {
            atomicExch(&status[tile], ep | ((unsigned long long)SCAN_AGG << 32) | (unsigned)agg);
            const unsigned long long t0 = story_clock_ns();
            bool late = false;
            for (int k = tile - 1; k >= 0;) {
                const unsigned long long w = atomicAdd(&status[k], 0ull);
                const unsigned fl = (unsigned)(w >> 32) & 3u;
                if ((w >> 34) != (unsigned long long)epoch || fl == 0) {
                    if (story_clock_ns() - t0 > kScanWaitNs) {
                        late = true;
                        break;
                    }
                    continue;
                }
                prefix += (int)(unsigned)w;
                if (fl == SCAN_PREFIX) break;
                --k;
            }
            if (late) report(err, 0, E_SCAN);
        }
        atomicExch(&status[tile], ep | ((unsigned long long)SCAN_PREFIX << 32) | (unsigned)(prefix + agg));
        if (tile == ntiles - 1 && total) *total = prefix + agg;
        s_prefix = prefix;
    }
    __syncthreads();
    int run = s_prefix + excl;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const int i = threadIdx.x * 16 + j;
        sv[i + i / 32] = run;
        run += v[j];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const int i = j * 256 + threadIdx.x;
        if (b + i < n) out[b + i] = sv[i + i / 32];
    }
}

// ---------------------------------------------------------------------------
// 1. Newline index.

// A block covers kNlTile bytes as kNlBytes / 16 rounds of 16-byte chunks:
// in round r thread t takes chunk r * kNlThreads + t (consecutive threads,
// consecutive chunks: coalesced).  Bytes past len read as zero.
__device__ __forceinline__ uint4 load16(const char *text, long long len, long long a) {
    if (a + 16 <= len) return *reinterpret_cast<const uint4 *>(text + a);
    uint32_t x[4] = {0, 0, 0, 0};
    for (int b = 0; b < 16; ++b)
        if (a + b < len) x[b >> 2] |= (uint32_t)(unsigned char)text[a + b] << (8 * (b & 3));
    return make_uint4(x[0], x[1], x[2], x[3]);
}

// Newline bits (bit b: byte b is '\n') and whether a NUL byte is present,
// for the 16 bytes of a chunk ending `left` bytes before len.
__device__ __forceinline__ uint32_t nl_bits16(uint4 q, long long left, bool &nul) {
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
    uint32_t bits = 0, zero = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t m = __vcmpeq4(w[k], 0x0a0a0a0au), z = __vcmpeq4(w[k], 0u);
        bits |= (((m >> 7) & 1u) | ((m >> 14) & 2u) | ((m >> 21) & 4u) | ((m >> 28) & 8u)) << (4 * k);
        zero |= (((z >> 7) & 1u) | ((z >> 14) & 2u) | ((z >> 21) & 4u) | ((z >> 28) & 8u)) << (4 * k);
    }
    const uint32_t keep = left >= 16 ? 0xffffu : (left <= 0 ? 0u : (1u << left) - 1u);
    nul |= (zero & keep) != 0;
    return bits & keep;
}

__global__ void __launch_bounds__(kNlThreads) nl_count_kernel(const char *text, long long len, long long *blk,
                                                              unsigned long long *err) {
    const long long base = (long long)blockIdx.x * kNlTile;
    int nl = 0;
    bool nul = false;
    uint4 q[kNlBytes / 16];
    if (base + kNlTile <= len) {  // all loads in flight before any is used
#pragma unroll
        for (int r = 0; r < kNlBytes / 16; ++r)
            q[r] = *reinterpret_cast<const uint4 *>(text + base + 16LL * (r * kNlThreads + threadIdx.x));
    } else {
#pragma unroll
        for (int r = 0; r < kNlBytes / 16; ++r) q[r] = load16(text, len, base + 16LL * (r * kNlThreads + threadIdx.x));
    }
#pragma unroll
    for (int r = 0; r < kNlBytes / 16; ++r) {
        const long long a = base + 16LL * (r * kNlThreads + threadIdx.x);
        if (a < len) nl += __popc(nl_bits16(q[r], len - a, nul));
    }
    if (nul) report(err, 0, E_NUL);
    int tot;
    block_excl_sum<kNlThreads>(nl, &tot);
    if (threadIdx.x == 0) blk[blockIdx.x] = (long long)tot;
}

__global__ void __launch_bounds__(kNlThreads) nl_write_kernel(const char *text, long long len,
                                                              const long long *blk_off, long long *nl_pos) {
    const long long base = (long long)blockIdx.x * kNlTile;
    long long o = blk_off[blockIdx.x];
    bool nul = false;
    uint4 q[kNlBytes / 16];
    if (base + kNlTile <= len) {
#pragma unroll
        for (int r = 0; r < kNlBytes / 16; ++r)
            q[r] = *reinterpret_cast<const uint4 *>(text + base + 16LL * (r * kNlThreads + threadIdx.x));
    } else {
#pragma unroll
        for (int r = 0; r < kNlBytes / 16; ++r) q[r] = load16(text, len, base + 16LL * (r * kNlThreads + threadIdx.x));
    }
#pragma unroll
    for (int r = 0; r < kNlBytes / 16; ++r) {
        const long long a = base + 16LL * (r * kNlThreads + threadIdx.x);
        uint32_t bits = a < len ? nl_bits16(q[r], len - a, nul) : 0u;
        int tot;
        long long at = o + block_excl_sum<kNlThreads>(__popc(bits), &tot);
        while (bits) {
            nl_pos[at++] = a + (__ffs(bits) - 1);
            bits &= bits - 1;
        }
        o += tot;
    }
}

// counts: [0] newlines, [1] lines, [2] last line unterminated; the same in
// meta[8..10], and meta[0] (end of the snapshot list) starts at the line
// count.  meta[11] = 1 when there are 2^31 - 2 lines or more (not read).
__global__ void line_count_kernel(const char *text, long long len, const long long *nnl, int *counts, int *meta) {
    const long long n64 = *nnl;
    const bool unterminated = len > 0 && text[len - 1] != '\n';
    const bool too_many = n64 >= 0x7ffffffdLL;
    const int n = too_many ? 0 : (int)n64;
    meta[11] = too_many;
    counts[0] = meta[8] = n;
    counts[1] = meta[9] = too_many ? 0 : n + (unterminated ? 1 : 0);
    counts[2] = meta[10] = unterminated;
    meta[0] = counts[1];
}

// ---------------------------------------------------------------------------
// 2. Classify every line.

__device__ __forceinline__ bool c_space(char c) { return c == ' ' || (c >= '\t' && c <= '\r'); }
__device__ __forceinline__ bool c_alnum(char c) {
    return (c >= '0' && c <= '9') || (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z');
}

__device__ __forceinline__ bool kw_is(const char *k, int n, const char *lit) {
    int i = 0;
    for (; i < n; ++i)
        if (lit[i] != k[i]) return false;
    return lit[i] == 0;
}

__device__ int keyword_id(const char *k, int n) {
    if (n == 1) {
        if (k[0] == 'm') return K_M;
        if (k[0] == 'r') return K_R;
        if (k[0] == 'v') return K_V;
        if (k[0] == 'i') return K_I;
        if (k[0] == 'N') return K_N;
        return K_OTHER;
    }
    if (kw_is(k, n, "system_time")) return K_TIME;
    if (kw_is(k, n, "real_system_time")) return K_RTIME;
    if (kw_is(k, n, "name")) return K_NAME;
    return K_OTHER;
}

__global__ void classify_kernel(const char *text, LineRange lr, const int *counts, uint32_t *tag) {
    const int nlines = counts[1];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nlines) return;
    long long s, e;
    lr.get(k, s, e);
    const long long full = e - s;
    const int n = (int)min(full, (long long)kLineMax);
    const char *l = text + s;
    uint32_t t = 0;
    if (n == 0) t |= F_EMPTY;
    if (full > kLineMax) t |= F_LONG;
    int j = 0;
    while (j < n && (signed char)l[j] <= ' ') ++j;
    if (j < n && (l[j] == '(' || l[j] == ')')) {
        if (j > 0) {
            t |= C_INDENT;
        } else {
            t |= l[0] == '(' ? C_OPEN : C_CLOSE;
            t |= (uint32_t)(n >= 2 ? (unsigned char)l[1] : 0u) << 8;
        }
    } else {
        int a = 0;
        while (a < n && c_space(l[a])) ++a;
        const int kb = a;
        while (a < n && (c_alnum(l[a]) || l[a] == '_')) ++a;
        const int ke = a;
        while (a < n && l[a] != '=') ++a;
        if (a < n) {
            ++a;
            while (a < n && c_space(l[a])) ++a;
            t |= C_KEY | ((uint32_t)keyword_id(l + kb, ke - kb) << 8) | ((uint32_t)a << 16);
        }
    }
    tag[k] = t;
}

struct DeltaF {
    const uint32_t *tag;
    __device__ int operator()(long long k) const { return delta_of(tag[k]); }
};

// 3. End of the snapshot list; structural checks up to it.  meta: [0] end
// line, [1] deepest level, [2] nodes, [3] roots, [4] leaves, [5] parents,
// [6] deepest node level.
__global__ void end_kernel(const uint32_t *tag, const int *depth, const int *counts, int *meta) {
    const int nlines = counts[1];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nlines) return;
    const uint32_t t = tag[k];
    if (depth[k] != 0) return;
    if ((t & F_EMPTY) || (k == nlines - 1 && counts[2] && code_of(t) != C_OPEN)) atomicMin(&meta[0], k);
}

__global__ void check_kernel(const uint32_t *tag, const int *depth, const int *counts, const int *depth_total,
                             int *meta, unsigned long long *err) {
    const int end = min(meta[0], counts[1]);
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0 && end >= counts[1] && *depth_total != 0) report(err, counts[1], E_EOF);
    int level = 0;
    if (k < end) {
        const uint32_t t = tag[k];
        const uint32_t c = code_of(t);
        const int d = depth[k];
        if (c == C_INDENT) report(err, k + 1, E_INDENT);
        if (d == 0 && c == C_CLOSE) report(err, k + 1, E_CLOSE0);
        if (d == 0 && c != C_OPEN && c != C_CLOSE) report(err, k + 1, E_TOP);
        if (d == 0 && c == C_OPEN && kind_of(t) != 'P') report(err, k + 1, E_TOP);
        if (c == C_OPEN) {
            if (d + 1 > kMaxDepth) report(err, k + 1, E_DEPTH);
            level = min(max(d + 1, 0), kMaxDepth);
        }
    }
    __shared__ int wl[8];  // blocks of 256: one atomic per block
    level = __reduce_max_sync(0xffffffffu, level);
    if ((threadIdx.x & 31) == 0) wl[threadIdx.x >> 5] = level;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < 8; ++i) level = max(level, wl[i]);
        if (level > 0) atomicMax(&meta[1], level);
    }
}

// ---------------------------------------------------------------------------
// 4. Enclosing open line of every line.

// Blocks of kChunkThreads chunks: each chunk's last open line per level,
// and the block's maximum per level (blk) for the scan across blocks.
// The block's lines are staged in shared memory by coalesced loads, stored
// chunk-transposed (line j of chunk c at j * kStageCols + c, kStageCols odd)
// so that the 32 threads of a warp, walking their chunks in step, read 32
// different banks.
constexpr int kChunkThreads = 128;
constexpr int kStageCols = kChunkThreads + 1;

__device__ __forceinline__ int staged(int i) { return (i % kChunk) * kStageCols + i / kChunk; }

__global__ void __launch_bounds__(kChunkThreads) chunk_last_kernel(const uint32_t *tag, const int *depth,
                                                                   const int *meta, int nchunks, int *sum, int *blk) {
    __shared__ int red[kChunkThreads / 32];
    __shared__ uint32_t s_tag[kChunk * kStageCols];
    __shared__ int s_dep[kChunk * kStageCols];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int end = meta[0], L = meta[1];
    const int b0 = blockIdx.x * kChunkThreads * kChunk;
    const int cnt = max(0, min(end - b0, kChunkThreads * kChunk));
    for (int i = threadIdx.x; i < cnt; i += kChunkThreads) {
        s_tag[staged(i)] = tag[b0 + i];
        s_dep[staged(i)] = depth[b0 + i];
    }
    __syncthreads();
    int last[kMaxDepth];
    for (int l = 0; l < L; ++l) last[l] = -1;
    if (c < nchunks) {
        const int b = c * kChunk, e = min(end, b + kChunk);
        for (int k = b; k < e; ++k) {
            const int i = staged(k - b0);
            if (code_of(s_tag[i]) == C_OPEN) {
                const int lv = s_dep[i] + 1;  // level of this open line (below 1 only in malformed text)
                if (lv >= 1 && lv <= kMaxDepth) last[lv - 1] = k;
            }
        }
        for (int l = 0; l < L; ++l) sum[(long long)c * kMaxDepth + l] = last[l];
    }
    for (int l = 0; l < L; ++l) {
        int m = __reduce_max_sync(0xffffffffu, last[l]);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int i = 1; i < kChunkThreads / 32; ++i) m = max(m, red[i]);
            m = max(m, red[0]);
            blk[(long long)blockIdx.x * kMaxDepth + l] = m;
        }
        __syncthreads();
    }
}

// Exclusive max-scan, per level, over n rows of kMaxDepth entries (one block).
__global__ void __launch_bounds__(1024) chunk_scan_kernel(int *sum, int nchunks, const int *meta) {
    const int L = meta[1];
    const int per = (nchunks + 1023) / 1024;
    const int b = threadIdx.x * per, e = min(nchunks, b + per);
    for (int l = 0; l < L; ++l) {
        int m = -1;
        for (int c = b; c < e; ++c) m = max(m, sum[(long long)c * kMaxDepth + l]);
        int run = block_excl_max<1024>(m);
        for (int c = b; c < e; ++c) {
            const int x = sum[(long long)c * kMaxDepth + l];
            sum[(long long)c * kMaxDepth + l] = run;
            run = max(run, x);
        }
    }
}

// blk holds, per block and level, the last open line before the block (an
// exclusive scan of chunk_last_kernel's maxima); the chunks of the block
// scan their own maxima to get the open lines around their start.  Tags
// in and enclosing lines out go through shared memory (staged()).
__global__ void __launch_bounds__(kChunkThreads) resolve_kernel(const uint32_t *tag, const int *depth, const int *meta,
                                                                int nchunks, const int *sum, const int *blk, int *encl) {
    __shared__ uint32_t s_tag[kChunk * kStageCols];
    __shared__ int s_enc[kChunk * kStageCols];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int end = meta[0], L = meta[1];
    const int b0 = blockIdx.x * kChunkThreads * kChunk;
    const int cnt = max(0, min(end - b0, kChunkThreads * kChunk));
    for (int i = threadIdx.x; i < cnt; i += kChunkThreads) s_tag[staged(i)] = tag[b0 + i];
    int st[kMaxDepth + 1];
    st[0] = -1;
    for (int l = 1; l <= L; ++l) {
        const int v = c < nchunks ? sum[(long long)c * kMaxDepth + l - 1] : -1;
        st[l] = max(block_excl_max<kChunkThreads>(v), blk[(long long)blockIdx.x * kMaxDepth + l - 1]);
    }
    __syncthreads();
    if (c < nchunks) {
        const int b = c * kChunk, e = min(end, b + kChunk);
        int d = b < e ? depth[b] : 0;
        for (int k = b; k < e; ++k) {
            const int i = staged(k - b0);
            const uint32_t code = code_of(s_tag[i]);
            const int dd = min(max(d, 0), kMaxDepth);
            s_enc[i] = st[dd];
            if (code == C_OPEN) {
                if (d + 1 <= kMaxDepth && d >= 0) st[d + 1] = k;
                ++d;
            } else if (code == C_CLOSE) {
                --d;
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < cnt; i += kChunkThreads) encl[b0 + i] = s_enc[staged(i)];
}

// ---------------------------------------------------------------------------
// 5. Context of the open lines: sections and chapters.

__device__ __forceinline__ bool section_kind(int kd) {
    return kd == 'P' || kd == 'D' || kd == 'H' || kd == 'S' || kd == 'L';
}

// ctx[k] for an open line: the nearest enclosing section line (-1: top).
__global__ void context_kernel(uint32_t *tag, const int *encl, const int *meta, int *ctx,
                               unsigned long long *err) {
    const int end = meta[0];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= end) return;
    const uint32_t t = tag[k];
    if (code_of(t) != C_OPEN) return;
    int chain[kMaxDepth];
    int m = 0;
    for (int a = encl[k]; a >= 0 && m < kMaxDepth; a = encl[a]) chain[m++] = a;
    // top-down: which ancestors are sections
    int cl = -1, ck = 0;  // current context line and kind (0: top)
    for (int i = m - 1; i >= -1; --i) {
        const int a = i >= 0 ? chain[i] : k;
        const int kd = kind_of(i >= 0 ? tag[a] : t);
        const bool sec = (ck == 0 || ck == 'P') && section_kind(kd);
        if (i < 0) {
            ctx[k] = cl;
            if (sec) {
                tag[k] = t | F_STRUCT;
            } else if ((ck == 'D' || ck == 'H' || ck == 'S') && kd == ck) {
                report(err, k + 1, E_CONFLICT);
            }
        } else if (sec) {
            cl = a;
            ck = kd;
        }
    }
}

struct NodeFlagF {
    const uint32_t *tag;
    const int *meta;
    __device__ int operator()(long long k) const {
        const uint32_t t = tag[k];
        return k < meta[0] && code_of(t) == C_OPEN && (t & F_STRUCT) && kind_of(t) == 'P';
    }
};

// ---------------------------------------------------------------------------
// 6-7. Nodes, their fields, and the line checks.

struct Nodes {
    int *line, *parent, *size, *index, *name_len, *win, *level;
    long long *name_off;
    double *mass, *pos, *vel, *shift;
    int *shifted;
};

__global__ void node_fill_kernel(const uint32_t *tag, const int *encl, const int *ctx, const int *nid,
                                 const int *meta, Nodes N) {
    const int end = meta[0];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= end) return;
    const uint32_t t = tag[k];
    const uint32_t c = code_of(t);
    if (c == C_OPEN && (t & F_STRUCT) && kind_of(t) == 'P') {
        const int id = nid[k];
        N.line[id] = k;
        N.parent[id] = ctx[k] >= 0 ? nid[ctx[k]] : -1;
        N.index[id] = -1;
        N.name_off[id] = -1;
        N.name_len[id] = 0;
        N.mass[id] = 1.0;
        for (int q = 0; q < 3; ++q) N.pos[3 * id + q] = N.vel[3 * id + q] = 0.0;
        for (int f = 0; f < FLD_COUNT; ++f) N.win[FLD_COUNT * id + f] = -1;
        N.shifted[id] = 0;
    } else if (c == C_CLOSE) {
        const int o = encl[k];
        if (o >= 0) {
            const uint32_t to = tag[o];
            if ((to & F_STRUCT) && kind_of(to) == 'P') N.size[nid[o]] = nid[k] - nid[o];
        }
    }
}

// The nearest enclosing section line of line k (-1: top).
__device__ __forceinline__ int section_of(const uint32_t *tag, const int *encl, int k) {
    int a = encl[k];
    for (int g = 0; a >= 0 && !(tag[a] & F_STRUCT) && g < kMaxDepth; ++g) a = encl[a];
    return a;
}

__global__ void lines_kernel(const char *text, LineRange lr, const uint32_t *tag, const int *encl, const int *ctx,
                             const int *nid, const int *meta, Nodes N, unsigned long long *err) {
    const int end = meta[0];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= end) return;
    const uint32_t t = tag[k];
    const uint32_t c = code_of(t);
    // the section holding this line (an open line's own context)
    const int sec = c == C_OPEN ? ctx[k] : section_of(tag, encl, k);
    const int sk = sec >= 0 ? kind_of(tag[sec]) : 0;
    const bool in_log = sk == 'L' && !(c == C_OPEN && (t & F_STRUCT));
    if (in_log && (t & F_LONG)) report(err, k + 1, E_LONG);
    if (in_log && (t & F_EMPTY)) report(err, k + 1, E_EMPTY);
    if (c == C_CLOSE) {
        const int o = encl[k];
        if (o < 0) return;
        const uint32_t to = tag[o];
        if (kind_of(to) != kind_of(t)) {
            report(err, k + 1, E_KIND);
            return;
        }
        // Log chapters: the whole title must match (get_chapter, story.C:192-198)
        const bool log_chapter = (to & F_STRUCT) ? kind_of(to) == 'L' : (ctx[o] >= 0 && kind_of(tag[ctx[o]]) == 'L');
        if (log_chapter) {
            long long so, sc;
            const int no = lr.span(o, so), nc = lr.span(k, sc);
            bool same = no == nc;
            for (int i = 1; same && i < no; ++i) same = text[so + i] == text[sc + i];
            if (!same) report(err, k + 1, E_TITLE);
        }
        return;
    }
    if (c != C_KEY) return;
    const int key = kind_of(t);
    if (sk == 'D') {
        const int owner = ctx[sec];  // the particle holding this Dynamics section
        const int id = nid[owner];
        int f = -1;
        if (key == K_M) f = FLD_M;
        else if (key == K_R) f = FLD_R;
        else if (key == K_V) f = FLD_V;
        else if (key == K_TIME) f = FLD_TIME;
        if (f >= 0) atomicMax(&N.win[FLD_COUNT * id + f], k);
    } else if (sk == 'P') {
        const int id = nid[sec];
        if (key == K_I) atomicMax(&N.win[FLD_COUNT * id + FLD_I], k);
        else if (key == K_NAME) atomicMax(&N.win[FLD_COUNT * id + FLD_NAME], k);
        else if (key != K_N) report(err, k + 1, E_KEYWORD);
    }
}

// A line staged in shared memory: 16-byte loads (single bytes past the
// text's end) of the aligned chunks covering it, stored as words into this
// thread's slot of kStageWords (an odd word count, so the 32 slots of a
// warp start on 32 different banks).  Returns the line's first byte in the
// slot, or the global pointer when the line does not fit.
constexpr int kStageWords = 29;  // 116 bytes: lines up to 100 bytes
__device__ __forceinline__ const char *stage_line(const char *text, long long len, long long s, int n,
                                                  uint32_t *slot) {
    const long long a0 = s & ~15LL;
    if (s + n - a0 > 4 * kStageWords) return text + s;
    for (long long a = a0; a < s + n; a += 16) {
        uint32_t *d = slot + (a - a0) / 4;
        if (a + 16 <= len) {
            const uint4 v = *reinterpret_cast<const uint4 *>(text + a);
            d[0] = v.x;
            d[1] = v.y;
            d[2] = v.z;
            d[3] = v.w;
        } else {
            for (int w = 0; w < 4; ++w) {
                uint32_t x = 0;
                for (int b = 0; b < 4; ++b) {
                    const long long o = a + 4 * w + b;
                    if (o < len) x |= (uint32_t)(unsigned char)text[o] << (8 * b);
                }
                d[w] = x;
            }
        }
    }
    return reinterpret_cast<const char *>(slot) + (s - a0);
}

__device__ bool read_vec(const char *l, int n, double *out) {
    int eq = 0;
    while (eq < n && l[eq] != '=') ++eq;
    const char *p = l + eq + 1, *e = l + n;
    story::Real a = story::parse_real(p, e);
    story::Real b = story::parse_real(p + a.n, e);
    story::Real c = story::parse_real(p + a.n + b.n, e);
    out[0] = a.v;
    out[1] = b.v;
    out[2] = c.v;
    return c.n > 0 && !a.err && !b.err && !c.err;
}

// One thread per (field, node), field-major so that a warp converts one
// kind of field: 0 mass, 1 position, 2 velocity, 3 index and name (mixing
// the fields in a warp measured 3x slower: the lanes diverge).
//
// The m, r and v lines are staged in shared memory first (a few 16-byte
// loads per line instead of a byte load per character).
__global__ void __launch_bounds__(256) values_kernel(const char *text, LineRange lr, const uint32_t *tag, int nnodes,
                                                     Nodes N, unsigned long long *err) {
    __shared__ uint32_t stage[256 * kStageWords];
    uint32_t *slot = stage + threadIdx.x * kStageWords;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4LL * nnodes) return;
    const int f = (int)(t / nnodes), id = (int)(t - (long long)f * nnodes);
    const int *w = N.win + FLD_COUNT * id;
    long long s;
    if (f == 0 && w[FLD_M] >= 0) {
        const int n = lr.span(w[FLD_M], s);
        const char *l = stage_line(text, lr.len, s, n, slot);
        const story::Real r = story::parse_real(l + voff_of(tag[w[FLD_M]]), l + n);
        if (r.err) report(err, w[FLD_M] + 1, E_NUMBER);
        N.mass[id] = r.v;
    }
    if (f == 1 && w[FLD_R] >= 0) {
        const int n = lr.span(w[FLD_R], s);
        if (!read_vec(stage_line(text, lr.len, s, n, slot), n, N.pos + 3 * id)) report(err, w[FLD_R] + 1, E_VECTOR);
    }
    if (f == 2 && w[FLD_V] >= 0) {
        const int n = lr.span(w[FLD_V], s);
        if (!read_vec(stage_line(text, lr.len, s, n, slot), n, N.vel + 3 * id)) report(err, w[FLD_V] + 1, E_VECTOR);
    }
    if (f == 3 && w[FLD_I] >= 0) {
        const int n = lr.span(w[FLD_I], s);
        const story::Long r = story::parse_long(text + s + voff_of(tag[w[FLD_I]]), text + s + n);
        N.index[id] = (int)(uint32_t)(uint64_t)r.v;  // long -> int, as the reference's assignment
    }
    if (f == 3 && w[FLD_NAME] >= 0) {
        const int n = lr.span(w[FLD_NAME], s), a = voff_of(tag[w[FLD_NAME]]);
        int b = a;
        while (b < n && !c_space(text[s + b])) ++b;
        N.name_off[id] = s + a;
        N.name_len[id] = b - a;
    }
}

// Node depth (root 0) and the roots / leaves / parents flags.
__global__ void node_level_kernel(int nnodes, Nodes N, int *meta) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nnodes) return;
    int lv = 0;
    for (int a = N.parent[id]; a >= 0 && lv < kMaxDepth; a = N.parent[a]) ++lv;
    N.level[id] = lv;
    if (N.size[id] > 1) atomicMax(&meta[6], lv);
}

struct RootF {
    const int *parent;
    __device__ int operator()(long long k) const { return parent[k] < 0; }
};
struct LeafF {
    const int *parent, *size;
    __device__ int operator()(long long k) const { return parent[k] >= 0 && size[k] == 1; }
};
struct ParentF {
    const int *size;
    __device__ int operator()(long long k) const { return size[k] > 1; }
};

__global__ void compact_kernel(long long n, const int *ex, const int *flag_src_parent,
                               const int *flag_src_size, int which, int *out) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    bool f;
    if (which == 0) f = flag_src_parent[k] < 0;
    else if (which == 1) f = flag_src_parent[k] >= 0 && flag_src_size[k] == 1;
    else f = flag_src_size[k] > 1;
    if (f) out[ex[k]] = (int)k;
}

// System time of each root: the last system_time line read up to its end
// (the reference's dyn::system_time is one static, dyn_io.C:30).
// The nodes holding a system_time line (few) raise their root's entry of
// root_line (indexed by node, -1 elsewhere) to that line.
__global__ void node_time_kernel(int nnodes, Nodes N, int *root_line) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nnodes) return;
    const int w = N.win[FLD_COUNT * id + FLD_TIME];
    if (w < 0) return;
    int r = id;
    for (int g = 0; N.parent[r] >= 0 && g < kMaxDepth; ++g) r = N.parent[r];
    atomicMax(&root_line[r], w);
}

__global__ void root_time_finish_kernel(const char *text, LineRange lr, const uint32_t *tag, const int *roots,
                                        int nroots, const int *root_line, double *root_time) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int run = -1;
    for (int r = 0; r < nroots; ++r) {
        run = max(run, root_line[roots[r]]);
        double t = 0.0;
        if (run >= 0) {
            long long s;
            const int n = lr.span(run, s);
            t = story::parse_real(text + s + voff_of(tag[run]), text + s + n).v;
        }
        root_time[r] = t;
    }
}

// ---------------------------------------------------------------------------
// 8. check_and_correct_node.  One warp per parent at this level: daughters
// are the nodes of its subtree whose parent it is, visited in id order; the
// warp stages 32 candidates at a time in shared memory and lanes 0-6 each
// carry one of the seven sums (m, m x, m y, m z, m vx, m vy, m vz) through
// them in order, with separately rounded products and sums.
constexpr int kCorrWarps = 4;
constexpr int kBigParent = 512;  // larger subtrees: correct_big_kernel
constexpr int kBigTile = 1024;
constexpr int kBigRow = kBigTile + 2;  // padded rows: 16-byte aligned, the seven lanes on different banks
constexpr size_t kBigSmem = sizeof(double) * 2 * 7 * kBigRow + sizeof(unsigned) * 2 * (kBigTile / 32);

__global__ void __launch_bounds__(32 * kCorrWarps) correct_level_kernel(const int *parents, int nparents, int level,
                                                                       int nnodes, Nodes N) {
    __shared__ double sv[kCorrWarps][7][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pi = blockIdx.x * kCorrWarps + w;
    if (pi >= nparents) return;
    const int p = parents[pi];
    if (N.level[p] != level || N.size[p] > kBigParent) return;
    const int end = min(p + N.size[p], nnodes);
    double acc = 0.0;
    for (int base = p + 1; base < end; base += 32) {
        const int d = base + lane;
        const bool dau = d < end && N.parent[d] == p;
        if (dau) {
            sv[w][0][lane] = N.mass[d];
            for (int q = 0; q < 3; ++q) {
                sv[w][1 + q][lane] = N.pos[3 * d + q];
                sv[w][4 + q][lane] = N.vel[3 * d + q];
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, dau);
        __syncwarp();
        if (lane < 7) {
            for (unsigned bits = m; bits; bits &= bits - 1) {
                const int j = __ffs(bits) - 1;
                const double mm = sv[w][0][j];
                acc = __dadd_rn(acc, lane == 0 ? mm : __dmul_rn(mm, sv[w][lane][j]));
            }
        }
        __syncwarp();
    }
    // lanes 0..6 hold m, p.x, p.y, p.z, v.x, v.y, v.z
    const double mtot = __shfl_sync(0xffffffffu, acc, 0);
    if (lane == 0) N.mass[p] = mtot;
    if (mtot > 0) {
        if (lane >= 1 && lane < 7) N.shift[6 * p + lane - 1] = __ddiv_rn(acc, mtot);
        if (lane == 0) N.shifted[p] = 1;
    }
}

// Parents with more than kBigParent candidates in their subtree (a
// snapshot root) take one block each: warps 1-7 stage the next tile of 1024
// candidates -- daughter flags and the seven addends (m and the separately
// rounded m x ... m vz) -- into shared memory while lanes 0-6 of warp 0 add
// the current tile's addends in order, full 32-candidate runs unrolled, so
// that the serial chain is one FP64 add per daughter.
__global__ void __launch_bounds__(256) correct_big_kernel(const int *parents, int nparents, int level, int nnodes,
                                                          Nodes N) {
    extern __shared__ __align__(16) double big_smem[];
    double(*add)[7][kBigRow] = reinterpret_cast<double(*)[7][kBigRow]>(big_smem);
    unsigned(*mask)[kBigTile / 32] = reinterpret_cast<unsigned(*)[kBigTile / 32]>(big_smem + 2 * 7 * kBigRow);
    const int pi = blockIdx.x;
    if (pi >= nparents) return;
    const int p = parents[pi];
    if (N.level[p] != level || N.size[p] <= kBigParent) return;
    const int end = min(p + N.size[p], nnodes);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = (end - (p + 1) + kBigTile - 1) / kBigTile;
    // stage tile t into buffer t & 1 using warps [w0, 8)
    auto stage = [&](int t, int w0) {
        const int nthr = (8 - w0) * 32, me = threadIdx.x - w0 * 32;
        const int b = t & 1, base = p + 1 + t * kBigTile;
        for (int i = me; i < kBigTile; i += nthr) {
            const int d = base + i;
            const bool dau = d < end && N.parent[d] == p;
            if (dau) {
                const double mm = N.mass[d];
                add[b][0][i] = mm;
                for (int q = 0; q < 3; ++q) {
                    add[b][1 + q][i] = __dmul_rn(mm, N.pos[3 * d + q]);
                    add[b][4 + q][i] = __dmul_rn(mm, N.vel[3 * d + q]);
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, dau);  // a warp stages 32 consecutive candidates
            if (lane == 0) mask[b][i >> 5] = m;
        }
    };
    stage(0, 0);
    __syncthreads();
    double acc = 0.0;
    for (int t = 0; t < ntiles; ++t) {
        if (w > 0) {
            if (t + 1 < ntiles) stage(t + 1, 1);
        } else if (lane < 7) {
            const int b = t & 1;
            const double *a = add[b][lane];
            for (int g = 0; g < kBigTile / 32; ++g) {
                const unsigned m = mask[b][g];
                if (m == 0xffffffffu) {
                    // all 32 addends into registers first, then the 32 dependent adds in order
                    const double2 *a2 = reinterpret_cast<const double2 *>(a + 32 * g);
                    double2 r[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) r[j] = a2[j];
                    asm volatile("" ::: "memory");  // keep the loads ahead of the dependent adds
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        acc = __dadd_rn(acc, r[j].x);
                        acc = __dadd_rn(acc, r[j].y);
                    }
                } else {
                    for (unsigned bits = m; bits; bits &= bits - 1) acc = __dadd_rn(acc, a[32 * g + __ffs(bits) - 1]);
                }
            }
        }
        __syncthreads();
    }
    if (w == 0) {
        const double mtot = __shfl_sync(0xffffffffu, acc, 0);
        if (lane == 0) N.mass[p] = mtot;
        if (mtot > 0) {
            if (lane >= 1 && lane < 7) N.shift[6 * p + lane - 1] = __ddiv_rn(acc, mtot);
            if (lane == 0) N.shifted[p] = 1;
        }
    }
}

__global__ void shift_kernel(int nnodes, Nodes N) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nnodes) return;
    const int p = N.parent[id];
    if (p < 0 || !N.shifted[p]) return;
    for (int q = 0; q < 3; ++q) {
        N.pos[3 * id + q] = __dadd_rn(N.pos[3 * id + q], -N.shift[6 * p + q]);
        N.vel[3 * id + q] = __dadd_rn(N.vel[3 * id + q], -N.shift[6 * p + 3 + q]);
    }
}

// 9. Leaves: positions and velocities relative to the root, summed from the
// leaf upwards starting at +0 as something_relative_to_root does.
__global__ void leaves_kernel(const int *leaves, int nleaves, Nodes N, double *lm, double *lx, double *lv, int *lidx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nleaves) return;
    const int id = leaves[i];
    double x[3] = {0.0, 0.0, 0.0}, v[3] = {0.0, 0.0, 0.0};
    for (int b = id; N.parent[b] >= 0; b = N.parent[b])
        for (int q = 0; q < 3; ++q) {
            x[q] = __dadd_rn(x[q], N.pos[3 * b + q]);
            v[q] = __dadd_rn(v[q], N.vel[3 * b + q]);
        }
    lm[i] = N.mass[id];
    for (int q = 0; q < 3; ++q) {
        lx[3 * i + q] = x[q];
        lv[3 * i + q] = v[q];
    }
    lidx[i] = N.index[id];
}

// ---------------------------------------------------------------------------
// Host side.

struct Buf {
    void *p = nullptr;
    size_t cap = 0;
};

class Reader {
  public:
    explicit Reader(int device) : device_(device) {}
    ~Reader() { release(); }
    std::string err;
    int open();
    int parse(const char *text, long long len, bool on_device, int flags, g6b200_story_info *info);
    long long n_nodes = 0, n_leaves = 0, n_roots = 0, bytes = 0, lines = 0;
    int max_depth = 0;
    Nodes N{};
    int *d_leaves = nullptr, *d_roots = nullptr, *d_lidx = nullptr;
    double *d_lm = nullptr, *d_lx = nullptr, *d_lv = nullptr, *d_rtime = nullptr;
    int device_;
    cudaStream_t stream = nullptr;
    int get_device(void *dst, const void *src, size_t bytes_);

  private:
    std::vector<Buf> bufs_;
    unsigned long long *d_ticket = nullptr;  // scan tile tickets, counting up across scans
    unsigned long long ticket_base_ = 0;
    unsigned scan_epoch_ = 0;
    int *d_meta = nullptr;
    unsigned long long *d_err = nullptr;
    int *h_meta = nullptr;
    unsigned long long *h_err = nullptr;
    template <class T>
    int ensure(int slot, T *&ptr, size_t count);
    void release();
    int fail(const char *what, cudaError_t e) {
        err = std::string("story: ") + what + ": " + cudaGetErrorString(e);
        return -1;
    }
    template <class F>
    int scan(F f, long long n, int *out, int *total, int slot);
    int sync_meta();
    int upload(const char *text, long long len, char *dst);
    // Host text upload: kUpThreads threads each stage slices of their part
    // of the text in two pinned slots of kUpSlice bytes and queue each
    // slice's copy on the stream as soon as it is staged.
    static constexpr int kUpThreads = 8;
    static constexpr size_t kUpSlice = 4u << 20;
    char *h_up_[kUpThreads][2] = {};
    cudaEvent_t ev_up_[kUpThreads][2] = {};
};

int Reader::upload(const char *text, long long len, char *dst) {
    cudaError_t e;
    if (len < (long long)kUpSlice) {  // small texts: one copy
        if ((e = cudaMemcpyAsync(dst, text, (size_t)len, cudaMemcpyHostToDevice, stream)) != cudaSuccess)
            return fail("text copy", e);
        return 0;
    }
    if (!h_up_[0][0]) {
        for (int t = 0; t < kUpThreads; ++t)
            for (int b = 0; b < 2; ++b) {
                if ((e = cudaMallocHost(&h_up_[t][b], kUpSlice)) != cudaSuccess) return fail("pinned memory", e);
                if ((e = cudaEventCreateWithFlags(&ev_up_[t][b], cudaEventDisableTiming)) != cudaSuccess)
                    return fail("event", e);
            }
    }
    const int nt = (int)std::min<long long>(kUpThreads, (len + (long long)kUpSlice - 1) / (long long)kUpSlice);
    cudaError_t errs[kUpThreads] = {};
    auto work = [&](int t) {
        const long long b0 = len * t / nt, b1 = len * (t + 1) / nt;
        int slot = 0;
        bool used[2] = {false, false};
        for (long long o = b0; o < b1; o += (long long)kUpSlice, slot ^= 1) {
            const size_t n = (size_t)std::min<long long>((long long)kUpSlice, b1 - o);
            cudaError_t r = cudaSuccess;
            if (used[slot]) r = cudaEventSynchronize(ev_up_[t][slot]);  // the slot's previous copy is done
            if (r == cudaSuccess) {
                memcpy(h_up_[t][slot], text + o, n);
                r = cudaMemcpyAsync(dst + o, h_up_[t][slot], n, cudaMemcpyHostToDevice, stream);
            }
            if (r == cudaSuccess) r = cudaEventRecord(ev_up_[t][slot], stream);
            if (r != cudaSuccess) {
                errs[t] = r;
                return;
            }
            used[slot] = true;
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(work, t);
    work(0);
    for (auto &x : th) x.join();
    for (int t = 0; t < nt; ++t)
        if (errs[t] != cudaSuccess) return fail("text copy", errs[t]);
    return 0;
}

enum Slot {
    S_TEXT, S_BLK, S_NLTOTAL, S_NL, S_TAG, S_DEPTH, S_ENCL, S_CTX, S_NID, S_CHUNK, S_CHUNKBLK, S_TILES, S_TILES2, S_COUNTS,
    S_NLINE, S_NPARENT, S_NSIZE, S_NINDEX, S_NNOFF, S_NNLEN, S_NWIN, S_NLEVEL, S_NMASS, S_NPOS, S_NVEL, S_NSHIFT,
    S_NSHIFTED, S_EX, S_ROOTS, S_LEAVES, S_PARENTS, S_LM, S_LX, S_LV, S_LIDX, S_RLINE, S_RTIME, S_COUNT
};

template <class T>
int Reader::ensure(int slot, T *&ptr, size_t count) {
    Buf &b = bufs_[slot];
    const size_t bytes_ = std::max<size_t>(count * sizeof(T), 256);
    if (bytes_ > b.cap) {
        if (b.p) cudaFree(b.p);
        b.p = nullptr;
        b.cap = 0;
        const size_t want = bytes_ + bytes_ / 4;
        cudaError_t e = cudaMalloc(&b.p, want);
        if (e != cudaSuccess) return fail("device memory", e);
        b.cap = want;
    }
    ptr = static_cast<T *>(b.p);
    return 0;
}

void Reader::release() {
    if (stream) cudaStreamSynchronize(stream);
    for (int t = 0; t < kUpThreads; ++t)
        for (int b = 0; b < 2; ++b) {
            if (h_up_[t][b]) cudaFreeHost(h_up_[t][b]);
            if (ev_up_[t][b]) cudaEventDestroy(ev_up_[t][b]);
            h_up_[t][b] = nullptr;
            ev_up_[t][b] = nullptr;
        }
    for (Buf &b : bufs_)
        if (b.p) cudaFree(b.p);
    bufs_.clear();
    if (d_meta) cudaFree(d_meta);
    if (d_err) cudaFree(d_err);
    if (d_ticket) cudaFree(d_ticket);
    if (h_meta) cudaFreeHost(h_meta);
    if (h_err) cudaFreeHost(h_err);
    if (stream) cudaStreamDestroy(stream);
    d_meta = nullptr;
    d_err = nullptr;
    h_meta = nullptr;
    h_err = nullptr;
    stream = nullptr;
}

int Reader::open() {
    cudaError_t e;
    if ((e = cudaSetDevice(device_)) != cudaSuccess) return fail("device", e);
    if ((e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)) != cudaSuccess) return fail("stream", e);
    bufs_.resize(S_COUNT);
    if ((e = cudaMalloc(&d_meta, 16 * sizeof(int))) != cudaSuccess) return fail("device memory", e);
    if ((e = cudaMalloc(&d_err, sizeof(unsigned long long))) != cudaSuccess) return fail("device memory", e);
    if ((e = cudaMalloc(&d_ticket, sizeof(unsigned long long))) != cudaSuccess) return fail("device memory", e);
    if ((e = cudaMemset(d_ticket, 0, sizeof(unsigned long long))) != cudaSuccess) return fail("device memory", e);
    if ((e = cudaMallocHost(&h_meta, 16 * sizeof(int))) != cudaSuccess) return fail("pinned memory", e);
    if ((e = cudaMallocHost(&h_err, sizeof(unsigned long long))) != cudaSuccess) return fail("pinned memory", e);
    if ((e = cudaFuncSetAttribute(correct_big_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBigSmem)) !=
        cudaSuccess)
        return fail("shared memory", e);
    return 0;
}

template <class F>
int Reader::scan(F f, long long n, int *out, int *total, int slot) {
    const int tiles = (int)std::max<long long>(1, (n + kScanTile - 1) / kScanTile);
    unsigned long long *st;
    const size_t cap_before = bufs_[slot].cap;
    if (ensure(slot, st, (size_t)tiles)) return -1;
    if (bufs_[slot].cap != cap_before) cudaMemsetAsync(st, 0, bufs_[slot].cap, stream);  // epoch 0: never current
    ++scan_epoch_;
    if (scan_epoch_ >= (1u << 30)) {  // the epoch field wrapped: start over on zeroed words
        scan_epoch_ = 1;
        cudaMemsetAsync(st, 0, bufs_[slot].cap, stream);
    }
    scan1_kernel<<<tiles, 256, 0, stream>>>(f, n, out, total, st, d_ticket, ticket_base_, scan_epoch_, tiles, d_err);
    ticket_base_ += (unsigned long long)tiles;
    return 0;
}

int Reader::sync_meta() {
    cudaMemcpyAsync(h_meta, d_meta, 16 * sizeof(int), cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(h_err, d_err, sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream);
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail("device execution", e);
    if (*h_err != ~0ull) {
        char buf[256];
        const long long line = (long long)(*h_err >> 8);
        snprintf(buf, sizeof buf, "story: line %lld: %s", line, error_text((int)(*h_err & 0xff)));
        err = buf;
        return -2;
    }
    return 0;
}

int Reader::parse(const char *text, long long len, bool on_device, int flags, g6b200_story_info *info) {
    if (!stream && open()) return -1;
    if (len < 0) {
        err = "story: negative text length";
        return -1;
    }
    cudaError_t e;
    if ((e = cudaSetDevice(device_)) != cudaSuccess) return fail("device", e);
    n_nodes = n_leaves = n_roots = 0;
    // text on the device, padded with zeros to the 64-byte loads
    const char *d_text;
    if (on_device) {
        if (((uintptr_t)text & 15) != 0) {
            err = "story: device text must be 16-byte aligned";
            return -1;
        }
        d_text = text;
    } else {
        char *t;
        if (ensure(S_TEXT, t, (size_t)len + 128)) return -1;
        if (len > 0 && upload(text, len, t)) return -1;
        d_text = t;
    }
    cudaMemsetAsync(d_err, 0xff, sizeof(unsigned long long), stream);
    cudaMemsetAsync(d_ticket, 0, sizeof(unsigned long long), stream);
    ticket_base_ = 0;
    const int init_meta[16] = {0x7fffffff, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    memcpy(h_meta, init_meta, sizeof init_meta);
    cudaMemcpyAsync(d_meta, h_meta, sizeof init_meta, cudaMemcpyHostToDevice, stream);
    // 1. newline index
    const int nblk = (int)std::max<long long>(1, (len + kNlTile - 1) / kNlTile);
    long long *blk, *nl, *nl_total;
    int *counts;
    if (ensure(S_BLK, blk, (size_t)nblk + 1) || ensure(S_COUNTS, counts, 8) || ensure(S_NLTOTAL, nl_total, 1))
        return -1;
    // a device text of unknown padding: read only [0, len) (the kernels stop at len; the vector loads of the
    // last 64-byte segment stay within the 16-byte-aligned allocation the caller was asked for)
    nl_count_kernel<<<nblk, kNlThreads, 0, stream>>>(d_text, len, blk, d_err);
    scan_tiles_kernel<<<1, 1024, 0, stream>>>(blk, nblk, nl_total);
    line_count_kernel<<<1, 1, 0, stream>>>(d_text, len, nl_total, counts, d_meta);
    if (sync_meta()) return -2;
    if (h_meta[11]) {
        err = "story: 2^31 - 2 lines or more (not read)";
        return -1;
    }
    const int nnl = h_meta[8], nlines = h_meta[9];
    lines = nlines;
    if (ensure(S_NL, nl, (size_t)nnl + 1)) return -1;
    nl_write_kernel<<<nblk, kNlThreads, 0, stream>>>(d_text, len, blk, nl);
    const LineRange lr{nl, nnl, len};
    // 2-3. classify, depth, end of the snapshot list, checks
    uint32_t *tag;
    int *depth, *encl, *ctx, *nid;
    if (ensure(S_TAG, tag, (size_t)nlines + 1) || ensure(S_DEPTH, depth, (size_t)nlines + 1) ||
        ensure(S_ENCL, encl, (size_t)nlines + 1) || ensure(S_CTX, ctx, (size_t)nlines + 1) ||
        ensure(S_NID, nid, (size_t)nlines + 1))
        return -1;
    const int lb = (nlines + 255) / 256;
    if (nlines > 0) {
        classify_kernel<<<lb, 256, 0, stream>>>(d_text, lr, counts, tag);
        if (scan(DeltaF{tag}, nlines, depth, counts + 5, S_TILES)) return -1;
        end_kernel<<<lb, 256, 0, stream>>>(tag, depth, counts, d_meta);
        check_kernel<<<lb, 256, 0, stream>>>(tag, depth, counts, counts + 5, d_meta, d_err);
    }
    // 4. enclosing lines
    const int nchunks = (nlines + kChunk - 1) / kChunk;
    int *chunk, *chunk_blk;
    const int cblocks = (nchunks + kChunkThreads - 1) / kChunkThreads;
    if (ensure(S_CHUNK, chunk, (size_t)std::max(nchunks, 1) * kMaxDepth) ||
        ensure(S_CHUNKBLK, chunk_blk, (size_t)std::max(cblocks, 1) * kMaxDepth))
        return -1;
    if (nchunks > 0) {
        chunk_last_kernel<<<cblocks, kChunkThreads, 0, stream>>>(tag, depth, d_meta, nchunks, chunk, chunk_blk);
        chunk_scan_kernel<<<1, 1024, 0, stream>>>(chunk_blk, cblocks, d_meta);
        resolve_kernel<<<cblocks, kChunkThreads, 0, stream>>>(tag, depth, d_meta, nchunks, chunk, chunk_blk, encl);
        // 5. sections and chapters
        context_kernel<<<lb, 256, 0, stream>>>(tag, encl, d_meta, ctx, d_err);
        // 6. node numbering
        if (scan(NodeFlagF{tag, d_meta}, nlines, nid, d_meta + 2, S_TILES)) return -1;
    }
    if (sync_meta()) return -2;
    const int end_line = std::min(h_meta[0], nlines);
    const int nn = h_meta[2];
    max_depth = h_meta[1];
    n_nodes = nn;
    {
        long long s_end = len > 0 ? len : 0;
        if (end_line < nlines) {
            // bytes up to the start of the line that ended the list
            long long nlpos = 0;
            if (end_line > 0 && get_device(&nlpos, nl + end_line - 1, sizeof(long long))) return -1;
            s_end = end_line > 0 ? nlpos + 1 : 0;
        }
        bytes = s_end;
    }
    if (nn > 0) {
        if (ensure(S_NLINE, N.line, nn) || ensure(S_NPARENT, N.parent, nn) || ensure(S_NSIZE, N.size, nn) ||
            ensure(S_NINDEX, N.index, nn) || ensure(S_NNOFF, N.name_off, nn) || ensure(S_NNLEN, N.name_len, nn) ||
            ensure(S_NWIN, N.win, (size_t)nn * FLD_COUNT) || ensure(S_NLEVEL, N.level, nn) ||
            ensure(S_NMASS, N.mass, nn) || ensure(S_NPOS, N.pos, (size_t)nn * 3) ||
            ensure(S_NVEL, N.vel, (size_t)nn * 3) || ensure(S_NSHIFT, N.shift, (size_t)nn * 6) ||
            ensure(S_NSHIFTED, N.shifted, nn))
            return -1;
        node_fill_kernel<<<lb, 256, 0, stream>>>(tag, encl, ctx, nid, d_meta, N);
        lines_kernel<<<lb, 256, 0, stream>>>(d_text, lr, tag, encl, ctx, nid, d_meta, N, d_err);
        const int nbk = (nn + 255) / 256;
        values_kernel<<<(int)((4LL * nn + 255) / 256), 256, 0, stream>>>(d_text, lr, tag, nn, N, d_err);
        node_level_kernel<<<nbk, 256, 0, stream>>>(nn, N, d_meta);
        int *ex;
        if (ensure(S_EX, ex, (size_t)nn * 3)) return -1;
        if (scan(RootF{N.parent}, nn, ex, d_meta + 3, S_TILES) ||
            scan(LeafF{N.parent, N.size}, nn, ex + nn, d_meta + 4, S_TILES2) ||
            scan(ParentF{N.size}, nn, ex + 2 * (size_t)nn, d_meta + 5, S_TILES))
            return -1;
        // the three scans reuse tile buffers in stream order
    }
    if (sync_meta()) return -2;
    n_roots = h_meta[3];
    n_leaves = h_meta[4];
    const int nparents = h_meta[5], top_level = h_meta[6];
    if (nn > 0) {
        int *ex = static_cast<int *>(bufs_[S_EX].p);
        const int nbk = (nn + 255) / 256;
        if (ensure(S_ROOTS, d_roots, (size_t)std::max<long long>(n_roots, 1)) ||
            ensure(S_LEAVES, d_leaves, (size_t)std::max<long long>(n_leaves, 1)))
            return -1;
        int *d_parents;
        if (ensure(S_PARENTS, d_parents, (size_t)std::max(nparents, 1))) return -1;
        compact_kernel<<<nbk, 256, 0, stream>>>(nn, ex, N.parent, N.size, 0, d_roots);
        compact_kernel<<<nbk, 256, 0, stream>>>(nn, ex + nn, N.parent, N.size, 1, d_leaves);
        compact_kernel<<<nbk, 256, 0, stream>>>(nn, ex + 2 * (size_t)nn, N.parent, N.size, 2, d_parents);
        int *rline;
        if (ensure(S_RLINE, rline, (size_t)nn) || ensure(S_RTIME, d_rtime, (size_t)std::max<long long>(n_roots, 1)))
            return -1;
        if (n_roots > 0) {
            cudaMemsetAsync(rline, 0xff, sizeof(int) * (size_t)nn, stream);
            node_time_kernel<<<nbk, 256, 0, stream>>>((int)nn, N, rline);
            root_time_finish_kernel<<<1, 32, 0, stream>>>(d_text, lr, tag, d_roots, (int)n_roots, rline, d_rtime);
        }
        if (!(flags & G6B200_STORY_RAW) && nparents > 0) {
            const int cb = (nparents + kCorrWarps - 1) / kCorrWarps;
            for (int lv = top_level; lv >= 0; --lv) {
                correct_level_kernel<<<cb, 32 * kCorrWarps, 0, stream>>>(d_parents, nparents, lv, (int)nn, N);
                correct_big_kernel<<<nparents, 256, kBigSmem, stream>>>(d_parents, nparents, lv, (int)nn, N);
            }
            shift_kernel<<<nbk, 256, 0, stream>>>(nn, N);
        }
        if (ensure(S_LM, d_lm, (size_t)std::max<long long>(n_leaves, 1)) ||
            ensure(S_LX, d_lx, (size_t)std::max<long long>(n_leaves, 1) * 3) ||
            ensure(S_LV, d_lv, (size_t)std::max<long long>(n_leaves, 1) * 3) ||
            ensure(S_LIDX, d_lidx, (size_t)std::max<long long>(n_leaves, 1)))
            return -1;
        if (n_leaves > 0)
            leaves_kernel<<<(int)((n_leaves + 255) / 256), 256, 0, stream>>>(d_leaves, (int)n_leaves, N, d_lm, d_lx,
                                                                           d_lv, d_lidx);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return fail("launch", e);
    if (sync_meta()) return -2;
    if (info) {
        info->bytes = bytes;
        info->lines = end_line;
        info->n_nodes = n_nodes;
        info->n_leaves = n_leaves;
        info->n_roots = n_roots;
        info->max_depth = max_depth;
    }
    return 0;
}

int Reader::get_device(void *dst, const void *src, size_t bytes_) {
    if (!bytes_) return 0;
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes_, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    return e == cudaSuccess ? 0 : fail("copy out", e);
}

}  // namespace storyk

// ---------------------------------------------------------------------------
// C ABI.

struct g6b200_story {
    storyk::Reader *r;
    bool parsed = false;
};

extern "C" {

g6b200_story *g6b200_story_create(int device) {
    auto *h = new g6b200_story{new storyk::Reader(device)};
    if (h->r->open()) {
        delete h->r;
        delete h;
        return nullptr;
    }
    return h;
}

void g6b200_story_destroy(g6b200_story *h) {
    if (!h) return;
    delete h->r;
    delete h;
}

const char *g6b200_story_error(g6b200_story *h) { return h ? h->r->err.c_str() : "story: null handle"; }

int g6b200_story_parse(g6b200_story *h, const char *text, long long len, int flags, g6b200_story_info *info) {
    if (!h || (!text && len > 0)) return -1;
    h->parsed = false;
    const int rc = h->r->parse(text, len, false, flags, info);
    h->parsed = rc == 0;
    return rc;
}

int g6b200_story_parse_device(g6b200_story *h, const char *d_text, long long len, int flags,
                              g6b200_story_info *info) {
    if (!h || (!d_text && len > 0)) return -1;
    h->parsed = false;
    const int rc = h->r->parse(d_text, len, true, flags, info);
    h->parsed = rc == 0;
    return rc;
}

int g6b200_story_nodes(g6b200_story *h, int *parent, int *index, double *mass, double (*pos)[3], double (*vel)[3]) {
    if (!h || !h->parsed) return -1;
    storyk::Reader &r = *h->r;
    const size_t n = (size_t)r.n_nodes;
    if (n == 0) return 0;
    if ((parent && r.get_device(parent, r.N.parent, 4 * n)) || (index && r.get_device(index, r.N.index, 4 * n)) ||
        (mass && r.get_device(mass, r.N.mass, 8 * n)) || (pos && r.get_device(pos, r.N.pos, 24 * n)) ||
        (vel && r.get_device(vel, r.N.vel, 24 * n)))
        return -1;
    return 0;
}

int g6b200_story_names(g6b200_story *h, long long *name_offset, int *name_length) {
    if (!h || !h->parsed) return -1;
    storyk::Reader &r = *h->r;
    const size_t n = (size_t)r.n_nodes;
    if (n == 0) return 0;
    if ((name_offset && r.get_device(name_offset, r.N.name_off, 8 * n)) ||
        (name_length && r.get_device(name_length, r.N.name_len, 4 * n)))
        return -1;
    return 0;
}

int g6b200_story_leaves(g6b200_story *h, int *node, int *index, double *mass, double (*pos)[3], double (*vel)[3]) {
    if (!h || !h->parsed) return -1;
    storyk::Reader &r = *h->r;
    const size_t n = (size_t)r.n_leaves;
    if (n == 0) return 0;
    if ((node && r.get_device(node, r.d_leaves, 4 * n)) || (index && r.get_device(index, r.d_lidx, 4 * n)) ||
        (mass && r.get_device(mass, r.d_lm, 8 * n)) || (pos && r.get_device(pos, r.d_lx, 24 * n)) ||
        (vel && r.get_device(vel, r.d_lv, 24 * n)))
        return -1;
    return 0;
}

int g6b200_story_roots(g6b200_story *h, int *root_node, double *system_time) {
    if (!h || !h->parsed) return -1;
    storyk::Reader &r = *h->r;
    const size_t n = (size_t)r.n_roots;
    if (n == 0) return 0;
    if ((root_node && r.get_device(root_node, r.d_roots, 4 * n)) ||
        (system_time && r.get_device(system_time, r.d_rtime, 8 * n)))
        return -1;
    return 0;
}

int g6b200_story_device_leaves(g6b200_story *h, const double **mass, const double **pos, const double **vel) {
    if (!h || !h->parsed) return -1;
    storyk::Reader &r = *h->r;
    if (mass) *mass = r.d_lm;
    if (pos) *pos = r.d_lx;
    if (vel) *vel = r.d_lv;
    return 0;
}

}  // extern "C"
