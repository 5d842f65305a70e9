// Eclipse INC and GSLIB property files on the GPU.
//
// Reading (read_inc_file.cpp:8-178).  The reference reads the property name
// line (read_prop_name), then `size` tokens with fscanf("%255s"): a token
// that starts with "--" skips the rest of its line, one that starts with '/'
// ends the data early (an error), every other token is one value, converted
// by sscanf("%f") or sscanf("%d").  Here the file is copied to the device
// once and every token is handled by its own thread:
//   1. tiles of 4096 bytes count the token starts and newlines of the data
//      section (k_tile_count), one block scans the tile counts
//      (k_scan_tiles), and the tiles write each token's start, end and line
//      number (k_tile_emit).  A token is a maximal run of non-blank bytes,
//      split every 255 bytes as "%255s" splits it (k_expand, only when a
//      longer run exists);
//   2. a token that starts with "--" marks its line (k_run_info): every later
//      token of that line is skipped, as "%*[^\n]" skips it;
//   3. the tokens that remain are values or '/'.  A block-wise prefix count
//      gives each value its index (k_count_values, k_scan_blocks), and each
//      thread converts its values in place (k_values) with the conversions
//      of numtext.cuh; the first token in file order that fails (a '/' or an
//      unparsable value before `size` values) is the error the reference
//      throws.
// The property name line is found on the host (it is the first line that
// starts with a letter), from the same host copy of the file.
//
// Writing (property_writer.cpp:18-214).  Each cell's line ("%E\n" or
// "%d\n") has a length known without formatting it; a block-wise prefix sum
// of the lengths places every line, and each thread formats its cells into
// the output text (k_format), which is copied back and written after the
// header.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/hpgl.h"
#include "engine.h"
#include "numtext.cuh"
#include "textio.h"

namespace hpgl_b200 {

#define TIO_CHECK(expr)                                                                              \
    do {                                                                                             \
        cudaError_t e__ = (expr);                                                                    \
        if (e__ != cudaSuccess)                                                                      \
            throw HpglError{HPGL_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e__)};     \
    } while (0)

namespace {

using namespace numtext;

constexpr int NT = 256;        // threads per block of every pass
constexpr int PER = 16;        // bytes, tokens or cells per thread
constexpr int BLK = NT * PER;  // items per block
constexpr unsigned FULL_MASK = 0xffffffffu;
constexpr unsigned long long F20 = (1ull << 20) - 1;  // packed 20-bit counters

enum : int { FLAG_LONG = 1, FLAG_COMMENT = 2, FLAG_BAD_REMAP = 4 };

// Exclusive block-wide scan of a 64-bit value; `total` is the block's sum.
template <int THREADS>
__device__ unsigned long long block_scan(unsigned long long v, unsigned long long &total) {
    __shared__ unsigned long long warp_sum[THREADS / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(FULL_MASK, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[w] = x;
    __syncthreads();
    unsigned long long base = 0, tot = 0;
#pragma unroll
    for (int i = 0; i < THREADS / 32; ++i) {
        const unsigned long long s = warp_sum[i];
        if (i < w) base += s;
        tot += s;
    }
    __syncthreads();
    total = tot;
    return base + x - v;
}

// The data section of the file on the device: bytes outside [begin, end)
// count as blanks.  The buffer holds at least BLK + 64 bytes past `end`.
struct Region {
    const unsigned char *txt;
    long long begin, end;
};

__device__ __forceinline__ bool blank(const Region &R, long long p, unsigned c) {
    return p < R.begin || p >= R.end || is_ws(c);
}

// The top bit of each byte of x gathered into bits 0..3.
__device__ __forceinline__ unsigned movemask4(unsigned x) { return ((x & 0x80808080u) * 0x00204081u) >> 28; }

// Bits 0..3: which bytes of w are one of " \t\n\v\f\r".
__device__ __forceinline__ unsigned blank4(unsigned w) {
    return movemask4(__vcmpeq4(w, 0x20202020u) | __vcmpltu4(__vsub4(w, 0x09090909u), 0x05050505u));
}

// One thread's 16 bytes as bit masks (bit j = byte pos0 + j): blanks
// (bytes outside the data section included), newlines inside it, and the
// blank state of the bytes just before and after.
struct Bytes16 {
    unsigned blank, nl;
    bool prev_blank, next_blank;
};

__device__ __forceinline__ Bytes16 scan16(const Region &R, long long pos0) {
    const uint4 v = *reinterpret_cast<const uint4 *>(R.txt + pos0);
    Bytes16 b;
    b.blank = blank4(v.x) | blank4(v.y) << 4 | blank4(v.z) << 8 | blank4(v.w) << 12;
    b.nl = movemask4(__vcmpeq4(v.x, 0x0a0a0a0au)) | movemask4(__vcmpeq4(v.y, 0x0a0a0a0au)) << 4 |
           movemask4(__vcmpeq4(v.z, 0x0a0a0a0au)) << 8 | movemask4(__vcmpeq4(v.w, 0x0a0a0a0au)) << 12;
    const long long lo = R.begin - pos0, hi = R.end - pos0;
    const int l = lo <= 0 ? 0 : (lo >= PER ? PER : (int)lo);
    const int h = hi <= 0 ? 0 : (hi >= PER ? PER : (int)hi);
    const unsigned inside = ((1u << h) - 1u) & ~((1u << l) - 1u);
    b.blank = (b.blank | ~inside) & 0xffffu;
    b.nl &= inside;
    // neighbours' edge bytes: from the lanes next door, else from memory
    const int lane = threadIdx.x & 31;
    const unsigned up = __shfl_up_sync(FULL_MASK, b.blank, 1);
    const unsigned down = __shfl_down_sync(FULL_MASK, b.blank, 1);
    b.prev_blank = lane ? (up >> 15) & 1u : (pos0 == 0 ? true : blank(R, pos0 - 1, R.txt[pos0 - 1]));
    b.next_blank = lane < 31 ? down & 1u : blank(R, pos0 + PER, R.txt[pos0 + PER]);
    return b;
}

// bit j: a run of non-blank bytes starts at byte j
__device__ __forceinline__ unsigned starts16(const Bytes16 &b) {
    return ~b.blank & ((b.blank << 1) | (b.prev_blank ? 1u : 0u)) & 0xffffu;
}
// bit j: a run ends with byte j
__device__ __forceinline__ unsigned ends16(const Bytes16 &b) {
    return ~b.blank & ((b.blank >> 1) | (b.next_blank ? 0x8000u : 0u)) & 0xffffu;
}

// Per tile: token starts (bits 0-19) and newlines (bits 20-39).
__global__ void __launch_bounds__(NT) k_tile_count(Region R, long long tile0, unsigned long long *tile_cnt) {
    const long long pos0 = (tile0 + blockIdx.x) * (long long)BLK + threadIdx.x * PER;
    const Bytes16 b = scan16(R, pos0);
    unsigned long long tot;
    block_scan<NT>((unsigned)__popc(starts16(b)) | ((unsigned long long)__popc(b.nl) << 20), tot);
    if (threadIdx.x == 0) tile_cnt[blockIdx.x] = tot;
}

// Exclusive prefix sums of the packed tile counts, one block; totals[0] =
// tokens (runs), totals[1] = newlines.
__global__ void __launch_bounds__(1024) k_scan_tiles(const unsigned long long *cnt, long long n, long long *run_base,
                                                     long long *nl_base, long long *totals) {
    const long long per = (n + 1023) / 1024;
    const long long a = threadIdx.x * per, b = min(n, a + per);
    unsigned long long s_runs = 0, s_nl = 0;
    for (long long i = a; i < b; ++i) {
        s_runs += cnt[i] & F20;
        s_nl += (cnt[i] >> 20) & F20;
    }
    unsigned long long t_runs, t_nl;
    unsigned long long r = block_scan<1024>(s_runs, t_runs);
    unsigned long long l = block_scan<1024>(s_nl, t_nl);
    for (long long i = a; i < b; ++i) {
        run_base[i] = (long long)r;
        nl_base[i] = (long long)l;
        r += cnt[i] & F20;
        l += (cnt[i] >> 20) & F20;
    }
    if (threadIdx.x == 0) {
        totals[0] = (long long)t_runs;
        totals[1] = (long long)t_nl;
    }
}

// Start, end (exclusive) and line number of every run of non-blank bytes.
// The runs that ended before a thread's first byte are the runs that started
// before it, less one when a run crosses into the thread's first byte.
__global__ void __launch_bounds__(NT) k_tile_emit(Region R, long long tile0, const long long *run_base,
                                                  const long long *nl_base, long long *run_start, long long *run_end,
                                                  long long *run_line) {
    const long long pos0 = (tile0 + blockIdx.x) * (long long)BLK + threadIdx.x * PER;
    const Bytes16 b = scan16(R, pos0);
    unsigned S = starts16(b), E = ends16(b);
    unsigned long long tot;
    const unsigned long long off =
        block_scan<NT>((unsigned)__popc(S) | ((unsigned long long)__popc(b.nl) << 20), tot);
    const long long si0 = run_base[blockIdx.x] + (long long)(off & F20);
    const long long line0 = nl_base[blockIdx.x] + (long long)((off >> 20) & F20);
    const bool open = !b.prev_blank && !(b.blank & 1u);
    long long si = si0, ei = si0 - (open ? 1 : 0);
    while (S) {
        const int j = __ffs(S) - 1;
        S &= S - 1;
        run_start[si] = pos0 + j;
        run_line[si] = line0 + __popc(b.nl & ((1u << j) - 1u));
        ++si;
    }
    while (E) {
        const int j = __ffs(E) - 1;
        E &= E - 1;
        run_end[ei] = pos0 + j + 1;
        ++ei;
    }
}

__device__ __forceinline__ bool is_comment_at(const unsigned char *txt, long long s, long long e) {
    return e - s >= 2 && txt[s] == '-' && txt[s + 1] == '-';
}

// Runs longer than 255 bytes (FLAG_LONG); otherwise the comment marks of
// the lines (FLAG_COMMENT), keyed by run index, which is then the token index.
__global__ void k_run_info(const unsigned char *txt, const long long *start, const long long *end,
                           const long long *line, long long n, long long *first_comment, int *flags) {
    const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (r >= n) return;
    const long long s = start[r], e = end[r];
    if (e - s > 255) atomicOr(flags, FLAG_LONG);
    if (is_comment_at(txt, s, e)) {
        atomicMin(first_comment + line[r], r);
        atomicOr(flags, FLAG_COMMENT);
    }
}

// Per block of runs: the number of 255-byte tokens they split into.
__global__ void __launch_bounds__(NT) k_count_chunks(const long long *start, const long long *end, long long n,
                                                     long long *block_sums) {
    const long long i0 = blockIdx.x * (long long)BLK + threadIdx.x * PER;
    unsigned long long cnt = 0;
    for (int j = 0; j < PER; ++j) {
        const long long r = i0 + j;
        if (r < n) cnt += (unsigned long long)((end[r] - start[r] + 254) / 255);
    }
    unsigned long long tot;
    block_scan<NT>(cnt, tot);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = (long long)tot;
}

// Exclusive scan of per-block sums in place, one block.
__global__ void __launch_bounds__(1024) k_scan_blocks(long long *v, long long n, long long *total) {
    const long long per = (n + 1023) / 1024;
    const long long a = threadIdx.x * per, b = min(n, a + per);
    unsigned long long s = 0;
    for (long long i = a; i < b; ++i) s += (unsigned long long)v[i];
    unsigned long long tot;
    unsigned long long r = block_scan<1024>(s, tot);
    for (long long i = a; i < b; ++i) {
        const long long x = v[i];
        v[i] = (long long)r;
        r += (unsigned long long)x;
    }
    if (threadIdx.x == 0) *total = (long long)tot;
}

// The 255-byte tokens of every run, with the comment marks keyed by token.
__global__ void __launch_bounds__(NT) k_expand(const unsigned char *txt, const long long *start, const long long *end,
                                               const long long *line, long long n, const long long *block_base,
                                               long long *tok_start, long long *tok_end, long long *tok_line,
                                               long long *first_comment, int *flags) {
    const long long i0 = blockIdx.x * (long long)BLK + threadIdx.x * PER;
    unsigned long long cnt = 0;
    for (int j = 0; j < PER; ++j) {
        const long long r = i0 + j;
        if (r < n) cnt += (unsigned long long)((end[r] - start[r] + 254) / 255);
    }
    unsigned long long tot;
    long long t = block_base[blockIdx.x] + (long long)block_scan<NT>(cnt, tot);
    for (int j = 0; j < PER; ++j) {
        const long long r = i0 + j;
        if (r >= n) break;
        for (long long s = start[r]; s < end[r]; s += 255, ++t) {
            const long long e = min(end[r], s + 255);
            tok_start[t] = s;
            tok_end[t] = e;
            tok_line[t] = line[r];
            if (is_comment_at(txt, s, e)) {
                atomicMin(first_comment + line[r], t);
                atomicOr(flags, FLAG_COMMENT);
            }
        }
    }
}

struct Tokens {
    const unsigned char *txt;
    const long long *start, *end, *line;
    const long long *first_comment;  // null when no token starts with "--"
    long long n;
};

// 0: skipped (a comment token or after one on its line), 1: value, 2: '/'
__device__ __forceinline__ int tok_class(const Tokens &T, long long t) {
    if (T.first_comment && T.first_comment[T.line[t]] <= t) return 0;
    return T.txt[T.start[t]] == '/' ? 2 : 1;
}

// Value tokens per block of NT tokens (one token per thread).
__global__ void __launch_bounds__(NT) k_count_values(Tokens T, long long *block_sums) {
    const long long t = blockIdx.x * (long long)NT + threadIdx.x;
    const int n = __syncthreads_count(t < T.n && tok_class(T, t) == 1);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = n;
}

struct ValueOut {
    long long size;  // values wanted
    int is_byte;
    int undefined_i;
    float *vals_f;
    unsigned char *vals_b;
    unsigned char *mask;  // byte reader: value != undefined
    unsigned long long *err_t, *err_vi;
    long long *last_read;  // last token the reference's scanner would read
};

// Converts every value token whose index is below `size`, one token per
// thread: a warp reads 32 neighbouring tokens of the text.
__global__ void __launch_bounds__(NT) k_values(Tokens T, const long long *block_base, ValueOut O) {
    const long long t = blockIdx.x * (long long)NT + threadIdx.x;
    const int cls = t < T.n ? tok_class(T, t) : 0;
    unsigned long long tot;
    const long long vi = block_base[blockIdx.x] + (long long)block_scan<NT>(cls == 1 ? 1u : 0u, tot);
    if (cls == 0 || vi >= O.size) return;
    if (cls == 2) {
        atomicMin(O.err_t, (unsigned long long)t);
        atomicMin(O.err_vi, (unsigned long long)vi);
        return;
    }
    const long long s = T.start[t];
    const unsigned char *p = T.txt + s;
    const int len = (int)(T.end[t] - s);
    // a token shorter than 255 bytes is a whole run, so a blank (or the
    // padding after the file) follows it: the unbounded conversions apply
    bool ok;
    if (O.is_byte) {
        int v;
        ok = len < 255 ? scan_int<false>(p, len, v) : scan_int<true>(p, len, v);
        if (ok) {
            O.vals_b[vi] = (unsigned char)v;
            O.mask[vi] = v == O.undefined_i ? 0 : 1;
        }
    } else {
        float v;
        ok = len < 255 ? scan_f32<false>(p, len, v) : scan_f32<true>(p, len, v);
        if (ok) O.vals_f[vi] = v;
    }
    if (!ok) {
        atomicMin(O.err_t, (unsigned long long)t);
        atomicMin(O.err_vi, (unsigned long long)vi);
    }
}

// The last token the reference's scanner reads: the last one that does not
// follow a comment mark on its line (only asked for when values run out).
__global__ void __launch_bounds__(NT) k_last_read(Tokens T, long long *last_read) {
    const long long t = blockIdx.x * (long long)NT + threadIdx.x;
    long long v = (t < T.n && (!T.first_comment || T.first_comment[T.line[t]] >= t)) ? t : -1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_down_sync(FULL_MASK, v, o));
    if ((threadIdx.x & 31) == 0 && v >= 0) atomicMax(last_read, v);
}

// A file with fewer values than asked: the reference's scanner keeps the
// last token it read in its buffer at end of file and converts it again for
// every remaining value.
__global__ void k_fill_tail(ValueOut O, long long from) {
    const long long i = from + blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= O.size) return;
    if (O.is_byte) {
        O.vals_b[i] = O.vals_b[from - 1];
        O.mask[i] = O.mask[from - 1];
    } else {
        O.vals_f[i] = O.vals_f[from - 1];
    }
}

// Float reader: informed = value != undefined (read_inc_file.cpp:145-153).
__global__ void k_float_mask(const float *v, unsigned char *mask, long long n, float undefined) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) mask[i] = v[i] == undefined ? 0 : 1;
}

// Byte reader: informed values replaced by the index of the first equal
// entry of `values` (api.cpp:84-98).
__global__ void k_remap(unsigned char *v, const unsigned char *mask, long long n, const unsigned char *values,
                        int count) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n || !mask[i]) return;
    const unsigned char x = v[i];
    for (int j = 0; j < count; ++j)
        if (values[j] == x) {
            v[i] = (unsigned char)j;
            return;
        }
}

// ---- writing -------------------------------------------------------------

struct Cells {
    const float *vf;
    const unsigned char *vb;
    const unsigned char *mask;
    long long n;
    int is_byte;
    float undefined_f;
    unsigned char undefined_b;
    const unsigned char *remap;
    int remap_count;
};

// The value a cell's line shows, and the line's length with its '\n'.
__device__ __forceinline__ int cell_line(const Cells &C, long long i, float &f, int &d, bool &bad) {
    bad = false;
    if (C.is_byte) {
        unsigned char x = C.undefined_b;
        if (C.mask[i]) {
            const unsigned char k = C.vb[i];
            if (k < C.remap_count) x = C.remap[k];
            else bad = true;
        }
        d = (int)(signed char)x;
        const int a = d < 0 ? -d : d;
        return (d < 0 ? 1 : 0) + (a >= 100 ? 3 : (a >= 10 ? 2 : 1)) + 1;
    }
    f = C.mask[i] ? C.vf[i] : C.undefined_f;
    const uint32_t u = f2u(f);
    return (int)(u >> 31) + ((u & 0x7fffffffu) >= 0x7f800000u ? 3 : 12) + 1;
}

// Text bytes per block of NT cells (one cell per thread).
__global__ void __launch_bounds__(NT) k_count_text(Cells C, long long *block_sums, int *flags) {
    const long long i = blockIdx.x * (long long)NT + threadIdx.x;
    unsigned len = 0;
    bool bad = false;
    if (i < C.n) {
        float f;
        int d;
        len = (unsigned)cell_line(C, i, f, d, bad);
    }
    if (bad) atomicOr(flags, FLAG_BAD_REMAP);
    unsigned long long tot;
    block_scan<NT>(len, tot);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = (long long)tot;
}

// One cell per thread; the block's lines are assembled in shared memory and
// stored with consecutive threads on consecutive bytes.
__global__ void __launch_bounds__(NT) k_format(Cells C, const long long *block_base, char *out) {
    __shared__ char text[NT * 16];
    const long long i = blockIdx.x * (long long)NT + threadIdx.x;
    char buf[16];
    int k = 0;
    if (i < C.n) {
        float f;
        int d;
        bool bad;
        cell_line(C, i, f, d, bad);
        k = C.is_byte ? format_d(d, buf) : format_E(f, buf);
        buf[k++] = '\n';
    }
    unsigned long long tot;
    const unsigned off = (unsigned)block_scan<NT>((unsigned)k, tot);
    for (int q = 0; q < k; ++q) text[off + q] = buf[q];
    __syncthreads();
    char *dst = out + block_base[blockIdx.x];
    for (unsigned q = threadIdx.x; q < (unsigned)tot; q += NT) dst[q] = text[q];
}

// ---- host side -------------------------------------------------------------

double ms_since(std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    template <typename T>
    T *get(size_t count) {
        const size_t bytes = std::max<size_t>(count * sizeof(T), 256);
        if (bytes > cap) {
            if (p) cudaFree(p);
            p = nullptr;
            cap = 0;
            const size_t want = bytes + bytes / 4;
            TIO_CHECK(cudaMalloc(&p, want));
            cap = want;
        }
        return static_cast<T *>(p);
    }
};

struct IoContext {
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    DevBuf text, tiles, run_base, nl_base, rs, re, rl, ts, te, tl, comment, blocks, small, vals, mask, values,
        cells_v, cells_m, remap, out;
    char *pinned = nullptr;
    size_t pinned_cap = 0;
    char *host(size_t bytes) {
        if (bytes > pinned_cap) {
            if (pinned) cudaFreeHost(pinned);
            pinned = nullptr;
            pinned_cap = 0;
            const size_t want = std::max<size_t>(bytes + bytes / 4, 1 << 20);
            TIO_CHECK(cudaHostAlloc((void **)&pinned, want, cudaHostAllocDefault));
            pinned_cap = want;
        }
        return pinned;
    }
};

std::mutex g_io_mutex;
TextIoTiming g_last_timing;  // guarded by g_io_mutex

IoContext &io_ctx() {
    static IoContext *c = nullptr;
    if (!c) {
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e == cudaSuccess && n == 0) e = cudaErrorNoDevice;
        if (e != cudaSuccess)
            throw HpglError{HPGL_E_CUDA, std::string("no CUDA device available: ") + cudaGetErrorString(e)};
        auto *nc = new IoContext();
        TIO_CHECK(cudaStreamCreateWithFlags(&nc->stream, cudaStreamNonBlocking));
        TIO_CHECK(cudaEventCreate(&nc->ev0));
        TIO_CHECK(cudaEventCreate(&nc->ev1));
        c = nc;
    }
    return *c;
}

unsigned grid_of(long long n, int per_block) { return (unsigned)std::max<long long>(1, (n + per_block - 1) / per_block); }

// Reads the whole file with a few threads (page-cache copies are bound by
// one core each).
void read_file(int fd, char *dst, size_t n) {
    const size_t slice_min = 8u << 20;
    const int nth = (int)std::max<size_t>(1, std::min<size_t>(8, n / slice_min));
    std::vector<std::thread> th;
    std::vector<int> failed(nth, 0);
    for (int k = 0; k < nth; ++k) {
        th.emplace_back([&, k] {
            size_t a = n * k / nth, b = n * (k + 1) / nth;
            while (a < b) {
                const ssize_t r = pread(fd, dst + a, b - a, (off_t)a);
                if (r <= 0) {
                    failed[k] = 1;
                    return;
                }
                a += (size_t)r;
            }
        });
    }
    for (auto &t : th) t.join();
    for (int f : failed)
        if (f) throw HpglError{HPGL_E_INVALID, "error reading the file"};
}

// Writes n bytes at offset `at` with a few threads.
void write_file(int fd, const char *src, long long n, long long at) {
    if (n <= 0) return;
    const long long slice_min = 8ll << 20;
    const int nth = (int)std::max<long long>(1, std::min<long long>(8, n / slice_min));
    std::vector<std::thread> th;
    std::vector<int> failed(nth, 0);
    for (int k = 0; k < nth; ++k) {
        th.emplace_back([&, k] {
            long long a = n * k / nth, b = n * (k + 1) / nth;
            while (a < b) {
                const ssize_t r = pwrite(fd, src + a, (size_t)(b - a), (off_t)(at + a));
                if (r <= 0) {
                    failed[k] = 1;
                    return;
                }
                a += r;
            }
        });
    }
    for (auto &t : th) t.join();
    for (int f : failed)
        if (f) throw HpglError{HPGL_E_INVALID, "error writing the file"};
}

// read_prop_name (read_inc_file.cpp:8-50): lines are read in pieces of up
// to 1023 bytes, each followed by a skip of all blanks; the first line whose
// first byte is a letter is the name, and data starts after it and the
// blanks that follow.  Two inputs on which the reference's loop never ends
// are errors here instead: a '\n' as the very first byte of the file is
// skipped as a blank line, and the end of the file right after a 1023-byte
// piece ends the search.
long long skip_header(const unsigned char *b, long long n) {
    long long p = 0;
    auto piece = [&](long long from) {
        long long q = from;
        while (q < n && b[q] != '\n' && q - from < 1023) ++q;
        return q;
    };
    auto skip_blanks = [&](long long q) {
        while (q < n && is_ws(b[q])) ++q;
        return q;
    };
    for (;;) {
        const long long q = piece(p);
        if (q == p) {
            if (p >= n) throw HpglError{HPGL_E_INVALID, "read_prop_name: Property name not found."};
            p = p + 1;  // a '\n' first in the file
            continue;
        }
        const unsigned c0 = b[p];
        const bool letter = (c0 - 'A') <= 25u || (c0 - 'a') <= 25u;
        long long len = q - p;
        p = skip_blanks(q);
        while (len == 1023) {
            if (p >= n) throw HpglError{HPGL_E_INVALID, "read_prop_name: Property name not found."};
            const long long q2 = piece(p);
            len = q2 - p;
            p = skip_blanks(q2);
        }
        if (letter) return p;
    }
}

std::string token_text(const unsigned char *b, long long s, long long e) {
    std::string t;
    for (long long i = s; i < e && b[i]; ++i) t += (char)b[i];
    return t;
}

}  // namespace

namespace {

// A file read into the pinned host buffer and split into tokens on the
// device.  `small` holds the pass counters: [0] runs, [1] newlines,
// [2] tokens, [3] values, [4] first failing token, [5] its value index,
// [6] last token read, [7] flags.
struct Tokenized {
    const unsigned char *h = nullptr;  // host copy of the file
    long long n = 0;                   // file size
    long long begin = 0;               // first byte after the name line
    Tokens T{};
    long long *small = nullptr;
};

Tokenized tokenize(IoContext &C, const char *filename, bool device, TextIoTiming &tm) {
    Tokenized K;
    const int fd = open(filename, O_RDONLY);
    if (fd < 0) throw HpglError{HPGL_E_INVALID, std::string("read_inc_file_float: Error opening file:") + filename + "."};
    struct FdCloser {
        int fd;
        ~FdCloser() { close(fd); }
    } closer{fd};
    struct stat st;
    if (fstat(fd, &st) != 0) throw HpglError{HPGL_E_INVALID, std::string("cannot stat ") + filename};
    const long long n = (long long)st.st_size;
    tm.bytes = n;
    cudaStream_t s = C.stream;
    auto t0 = std::chrono::steady_clock::now();
    unsigned char *h = (unsigned char *)C.host((size_t)n + 1);
    K.h = h;
    K.n = n;
    if (!device) {
        read_file(fd, (char *)h, (size_t)n);
        tm.ms_file = ms_since(t0);
        K.begin = skip_header(h, n);
        return K;
    }
    // the whole file with a few threads, then one copy to the device, padded
    // so that every tile reads whole 16-byte words past the end (a copy per
    // chunk as chunks arrive measured slower: page-cache reads and the DMA
    // share the host's memory bandwidth)
    read_file(fd, (char *)h, (size_t)n);
    tm.ms_file = ms_since(t0);
    K.begin = skip_header(h, n);
    const long long padded = n + 2 * BLK + 64;
    unsigned char *d_txt = C.text.get<unsigned char>((size_t)padded);
    t0 = std::chrono::steady_clock::now();
    TIO_CHECK(cudaMemcpyAsync(d_txt, h, (size_t)n, cudaMemcpyHostToDevice, s));
    TIO_CHECK(cudaMemsetAsync(d_txt + n, ' ', (size_t)(padded - n), s));
    TIO_CHECK(cudaStreamSynchronize(s));
    tm.ms_h2d = ms_since(t0);
    const long long tile0 = K.begin / BLK;
    const long long ntiles = std::max<long long>(1, (n - tile0 * BLK + BLK - 1) / BLK);

    TIO_CHECK(cudaEventRecord(C.ev0, s));
    const Region R{d_txt, K.begin, n};
    unsigned long long *d_tiles = C.tiles.get<unsigned long long>((size_t)ntiles);
    long long *d_run_base = C.run_base.get<long long>((size_t)ntiles);
    long long *d_nl_base = C.nl_base.get<long long>((size_t)ntiles);
    long long *d_small = C.small.get<long long>(8);
    K.small = d_small;
    TIO_CHECK(cudaMemsetAsync(d_small, 0, 8 * sizeof(long long), s));
    TIO_CHECK(cudaMemsetAsync(d_small + 4, 0xff, 3 * sizeof(long long), s));
    k_tile_count<<<(unsigned)ntiles, NT, 0, s>>>(R, tile0, d_tiles);
    k_scan_tiles<<<1, 1024, 0, s>>>(d_tiles, ntiles, d_run_base, d_nl_base, d_small);
    long long hs[2];
    TIO_CHECK(cudaMemcpyAsync(hs, d_small, 2 * sizeof(long long), cudaMemcpyDeviceToHost, s));
    TIO_CHECK(cudaStreamSynchronize(s));
    const long long runs = hs[0], lines = hs[1] + 1;

    long long *d_rs = C.rs.get<long long>((size_t)runs);
    long long *d_re = C.re.get<long long>((size_t)runs);
    long long *d_rl = C.rl.get<long long>((size_t)runs);
    long long *d_comment = C.comment.get<long long>((size_t)lines);
    int *d_flags = reinterpret_cast<int *>(d_small + 7);
    if (runs > 0) {
        k_tile_emit<<<(unsigned)ntiles, NT, 0, s>>>(R, tile0, d_run_base, d_nl_base, d_rs, d_re, d_rl);
        TIO_CHECK(cudaMemsetAsync(d_comment, 0x7f, (size_t)lines * sizeof(long long), s));
        k_run_info<<<grid_of(runs, 256), 256, 0, s>>>(d_txt, d_rs, d_re, d_rl, runs, d_comment, d_flags);
    }
    int flags = 0;
    TIO_CHECK(cudaMemcpyAsync(&flags, d_flags, sizeof(int), cudaMemcpyDeviceToHost, s));
    TIO_CHECK(cudaStreamSynchronize(s));

    const long long *ts = d_rs, *te = d_re, *tl = d_rl;
    long long ntok = runs;
    if (flags & FLAG_LONG) {
        const long long nb = (runs + BLK - 1) / BLK;
        long long *d_blocks = C.blocks.get<long long>((size_t)nb);
        k_count_chunks<<<(unsigned)nb, NT, 0, s>>>(d_rs, d_re, runs, d_blocks);
        k_scan_blocks<<<1, 1024, 0, s>>>(d_blocks, nb, d_small + 2);
        TIO_CHECK(cudaMemcpyAsync(&ntok, d_small + 2, sizeof(long long), cudaMemcpyDeviceToHost, s));
        TIO_CHECK(cudaStreamSynchronize(s));
        long long *d_ts = C.ts.get<long long>((size_t)ntok);
        long long *d_te = C.te.get<long long>((size_t)ntok);
        long long *d_tl = C.tl.get<long long>((size_t)ntok);
        TIO_CHECK(cudaMemsetAsync(d_comment, 0x7f, (size_t)lines * sizeof(long long), s));
        TIO_CHECK(cudaMemsetAsync(d_flags, 0, sizeof(int), s));
        k_expand<<<(unsigned)nb, NT, 0, s>>>(d_txt, d_rs, d_re, d_rl, runs, d_blocks, d_ts, d_te, d_tl, d_comment,
                                              d_flags);
        TIO_CHECK(cudaMemcpyAsync(&flags, d_flags, sizeof(int), cudaMemcpyDeviceToHost, s));
        TIO_CHECK(cudaStreamSynchronize(s));
        ts = d_ts;
        te = d_te;
        tl = d_tl;
    }
    tm.tokens = ntok;
    K.T = Tokens{d_txt, ts, te, tl, (flags & FLAG_COMMENT) ? d_comment : nullptr, ntok};
    return K;
}

// First '/' token that is not in a comment.
__global__ void k_first_slash(Tokens T, unsigned long long *first) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t < T.n && tok_class(T, t) == 2) atomicMin(first, (unsigned long long)t);
}

// Values before token `limit` (or all).
__global__ void k_count_before(Tokens T, const unsigned long long *limit, unsigned long long *count) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const bool v = t < T.n && (unsigned long long)t < *limit && tok_class(T, t) == 1;
    const unsigned b = __ballot_sync(FULL_MASK, v);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(count, (unsigned long long)__popc(b));
}

long long token_bound(const Tokens &T, long long t, bool end) {
    long long v = 0;
    TIO_CHECK(cudaMemcpy(&v, (end ? T.end : T.start) + t, sizeof(long long), cudaMemcpyDeviceToHost));
    return v;
}

}  // namespace

TextIoTiming last_io_timing() {
    std::lock_guard<std::mutex> lock(g_io_mutex);
    return g_last_timing;
}

void set_last_io_timing(const TextIoTiming &t) {
    std::lock_guard<std::mutex> lock(g_io_mutex);
    g_last_timing = t;
}

long long inc_count(const char *filename, bool is_byte, TextIoTiming *timing) {
    (void)is_byte;
    if (!filename) throw HpglError{HPGL_E_INVALID, "file name is null"};
    TextIoTiming tm;
    std::lock_guard<std::mutex> lock(g_io_mutex);
    IoContext &C = io_ctx();
    Tokenized K = tokenize(C, filename, true, tm);
    cudaStream_t s = C.stream;
    unsigned long long *first = reinterpret_cast<unsigned long long *>(K.small + 4);
    unsigned long long *count = reinterpret_cast<unsigned long long *>(K.small + 3);
    TIO_CHECK(cudaMemsetAsync(count, 0, sizeof(long long), s));
    if (K.T.n > 0) {
        k_first_slash<<<grid_of(K.T.n, 256), 256, 0, s>>>(K.T, first);
        k_count_before<<<grid_of(K.T.n, 256), 256, 0, s>>>(K.T, first, count);
    }
    long long c = 0;
    TIO_CHECK(cudaMemcpyAsync(&c, count, sizeof(long long), cudaMemcpyDeviceToHost, s));
    TIO_CHECK(cudaStreamSynchronize(s));
    g_last_timing = tm;
    if (timing) *timing = tm;
    return c;
}

void inc_read(const char *filename, bool is_byte, float undefined_f, int undefined_i, long long size, float *data_f,
              unsigned char *data_b, unsigned char *mask, const unsigned char *values, int values_count,
              TextIoTiming *timing) {
    const auto t_start = std::chrono::steady_clock::now();
    TextIoTiming tm;
    const char *where_data = is_byte ? "read_bytes" : "load_floats_into_vector";
    if (!filename) throw HpglError{HPGL_E_INVALID, "file name is null"};
    if (size > 0 && (!mask || (is_byte ? !data_b : !data_f)))
        throw HpglError{HPGL_E_INVALID, "output buffers are null"};
    if (is_byte && values_count > 0 && !values) throw HpglError{HPGL_E_INVALID, "values are null"};

    std::lock_guard<std::mutex> lock(g_io_mutex);
    IoContext &C = io_ctx();
    cudaStream_t s = C.stream;
    Tokenized K = tokenize(C, filename, size > 0, tm);
    if (size <= 0) {
        g_last_timing = tm;
    if (timing) *timing = tm;
        return;
    }
    const Tokens &T = K.T;
    const unsigned char *h = K.h;
    long long *d_small = K.small;
    ValueOut O;
    O.size = size;
    O.is_byte = is_byte ? 1 : 0;
    O.undefined_i = undefined_i;
    O.vals_f = is_byte ? nullptr : C.vals.get<float>((size_t)size);
    O.vals_b = is_byte ? C.vals.get<unsigned char>((size_t)size) : nullptr;
    O.mask = C.mask.get<unsigned char>((size_t)size);
    O.err_t = reinterpret_cast<unsigned long long *>(d_small + 4);
    O.err_vi = reinterpret_cast<unsigned long long *>(d_small + 5);
    O.last_read = d_small + 6;
    if (T.n > 0) {
        const long long nb = (T.n + NT - 1) / NT;
        long long *d_blocks = C.blocks.get<long long>((size_t)nb);
        k_count_values<<<(unsigned)nb, NT, 0, s>>>(T, d_blocks);
        k_scan_blocks<<<1, 1024, 0, s>>>(d_blocks, nb, d_small + 3);
        k_values<<<(unsigned)nb, NT, 0, s>>>(T, d_blocks, O);
    }
    long long hs[8];
    TIO_CHECK(cudaMemcpyAsync(hs, d_small, 8 * sizeof(long long), cudaMemcpyDeviceToHost, s));
    TIO_CHECK(cudaStreamSynchronize(s));
    const long long nvals = T.n > 0 ? hs[3] : 0;
    const unsigned long long err_t = (unsigned long long)hs[4], err_vi = (unsigned long long)hs[5];
    long long last_read = -1;
    if (err_t == ~0ull && nvals < size && T.n > 0) {
        k_last_read<<<grid_of(T.n, NT), NT, 0, s>>>(T, d_small + 6);
        TIO_CHECK(cudaMemcpyAsync(&last_read, d_small + 6, sizeof(long long), cudaMemcpyDeviceToHost, s));
        TIO_CHECK(cudaStreamSynchronize(s));
    }
    const size_t elem = is_byte ? 1 : 4;
    void *out_vals = is_byte ? (void *)O.vals_b : (void *)O.vals_f;
    void *user_vals = is_byte ? (void *)data_b : (void *)data_f;
    if (err_t != ~0ull) {
        // values before the failing token are stored, as the reference
        // stores them before it throws (and the byte reader's masks too)
        const long long keep = (long long)err_vi;
        if (keep > 0) {
            TIO_CHECK(cudaMemcpyAsync(user_vals, out_vals, (size_t)keep * elem, cudaMemcpyDeviceToHost, s));
            if (is_byte) TIO_CHECK(cudaMemcpyAsync(mask, O.mask, (size_t)keep, cudaMemcpyDeviceToHost, s));
            TIO_CHECK(cudaStreamSynchronize(s));
        }
        const long long ts = token_bound(T, (long long)err_t, false), te = token_bound(T, (long long)err_t, true);
        if (h[ts] == '/') throw HpglError{HPGL_E_INVALID, std::string(where_data) + ": Unexpected end of data."};
        throw HpglError{HPGL_E_INVALID,
                        std::string("load_floats_into_vector: Error parsing '") + token_text(h, ts, te) + "' string."};
    }
    if (nvals < size) {
        // end of file before `size` values: the last token read is converted
        // again; when there is none, or it is a comment (the reference's
        // loop never ends then), the data ended early
        bool repeat = false;
        if (last_read >= 0 && nvals > 0) {
            const long long ts = token_bound(T, last_read, false), te = token_bound(T, last_read, true);
            repeat = !(te - ts >= 2 && h[ts] == '-' && h[ts + 1] == '-');
        }
        if (!repeat) {
            if (nvals > 0) {  // the values read so far stay, as in the reference
                TIO_CHECK(cudaMemcpyAsync(user_vals, out_vals, (size_t)nvals * elem, cudaMemcpyDeviceToHost, s));
                if (is_byte) TIO_CHECK(cudaMemcpyAsync(mask, O.mask, (size_t)nvals, cudaMemcpyDeviceToHost, s));
                TIO_CHECK(cudaStreamSynchronize(s));
            }
            throw HpglError{HPGL_E_INVALID, std::string(where_data) + ": Unexpected end of data."};
        }
        k_fill_tail<<<grid_of(size - nvals, 256), 256, 0, s>>>(O, nvals);
    }
    if (is_byte) {
        if (values_count > 0) {
            unsigned char *d_values = C.values.get<unsigned char>((size_t)values_count);
            TIO_CHECK(cudaMemcpyAsync(d_values, values, (size_t)values_count, cudaMemcpyHostToDevice, s));
            k_remap<<<grid_of(size, 256), 256, 0, s>>>(O.vals_b, O.mask, size, d_values, values_count);
        }
    } else {
        k_float_mask<<<grid_of(size, 256), 256, 0, s>>>(O.vals_f, O.mask, size, undefined_f);
    }
    TIO_CHECK(cudaEventRecord(C.ev1, s));
    auto t0 = std::chrono::steady_clock::now();
    TIO_CHECK(cudaMemcpyAsync(user_vals, out_vals, (size_t)size * elem, cudaMemcpyDeviceToHost, s));
    TIO_CHECK(cudaMemcpyAsync(mask, O.mask, (size_t)size, cudaMemcpyDeviceToHost, s));
    TIO_CHECK(cudaStreamSynchronize(s));
    tm.ms_d2h = ms_since(t0);
    float ms = 0;
    cudaEventElapsedTime(&ms, C.ev0, C.ev1);
    tm.ms_device = ms;
    tm.ms_total = ms_since(t_start);
    g_last_timing = tm;
    if (timing) *timing = tm;
}

void prop_write(int format, bool is_byte, const char *filename, const char *name, const float *data_f,
                const unsigned char *data_b, const unsigned char *mask, long long size, float undefined_f,
                unsigned char undefined_b, const unsigned char *remap, int remap_count, TextIoTiming *timing) {
    const auto t_start = std::chrono::steady_clock::now();
    TextIoTiming tm;
    if (!filename || !name) throw HpglError{HPGL_E_INVALID, "file name or property name is null"};
    if (size < 0) size = 0;
    if (size > 0 && (!mask || (is_byte ? !data_b : !data_f))) throw HpglError{HPGL_E_INVALID, "data is null"};

    std::lock_guard<std::mutex> lock(g_io_mutex);
    IoContext &C = io_ctx();
    cudaStream_t s = C.stream;
    long long body = 0;
    char *h = nullptr;
    if (size > 0) {
        auto t0 = std::chrono::steady_clock::now();
        Cells X;
        X.n = size;
        X.is_byte = is_byte ? 1 : 0;
        X.undefined_f = undefined_f;
        X.undefined_b = undefined_b;
        X.remap_count = remap_count;
        unsigned char *d_m = C.cells_m.get<unsigned char>((size_t)size);
        TIO_CHECK(cudaMemcpyAsync(d_m, mask, (size_t)size, cudaMemcpyHostToDevice, s));
        X.mask = d_m;
        X.vf = nullptr;
        X.vb = nullptr;
        X.remap = nullptr;
        if (is_byte) {
            unsigned char *d_v = C.cells_v.get<unsigned char>((size_t)size);
            TIO_CHECK(cudaMemcpyAsync(d_v, data_b, (size_t)size, cudaMemcpyHostToDevice, s));
            X.vb = d_v;
            unsigned char *d_r = C.remap.get<unsigned char>(256);
            if (remap_count > 0)
                TIO_CHECK(cudaMemcpyAsync(d_r, remap, (size_t)remap_count, cudaMemcpyHostToDevice, s));
            X.remap = d_r;
        } else {
            float *d_v = C.cells_v.get<float>((size_t)size);
            TIO_CHECK(cudaMemcpyAsync(d_v, data_f, (size_t)size * 4, cudaMemcpyHostToDevice, s));
            X.vf = d_v;
        }
        TIO_CHECK(cudaStreamSynchronize(s));
        tm.ms_h2d = ms_since(t0);
        TIO_CHECK(cudaEventRecord(C.ev0, s));
        const long long nb = (size + NT - 1) / NT;
        long long *d_blocks = C.blocks.get<long long>((size_t)nb);
        long long *d_small = C.small.get<long long>(8);
        TIO_CHECK(cudaMemsetAsync(d_small, 0, 8 * sizeof(long long), s));
        int *d_flags = reinterpret_cast<int *>(d_small + 7);
        k_count_text<<<(unsigned)nb, NT, 0, s>>>(X, d_blocks, d_flags);
        k_scan_blocks<<<1, 1024, 0, s>>>(d_blocks, nb, d_small);
        long long hs[8];
        TIO_CHECK(cudaMemcpyAsync(hs, d_small, 8 * sizeof(long long), cudaMemcpyDeviceToHost, s));
        TIO_CHECK(cudaStreamSynchronize(s));
        if (((int *)(hs + 7))[0] & FLAG_BAD_REMAP)
            throw HpglError{HPGL_E_INVALID, "an informed value is outside the table of indicator values"};
        body = hs[0];
        char *d_out = C.out.get<char>((size_t)body);
        k_format<<<(unsigned)nb, NT, 0, s>>>(X, d_blocks, d_out);
        TIO_CHECK(cudaEventRecord(C.ev1, s));
        t0 = std::chrono::steady_clock::now();
        h = C.host((size_t)body);
        TIO_CHECK(cudaMemcpyAsync(h, d_out, (size_t)body, cudaMemcpyDeviceToHost, s));
        TIO_CHECK(cudaStreamSynchronize(s));
        tm.ms_d2h = ms_since(t0);
        float ms = 0;
        cudaEventElapsedTime(&ms, C.ev0, C.ev1);
        tm.ms_device = ms;
    }
    auto t0 = std::chrono::steady_clock::now();
    // fopen(filename, "w+") of the reference, then the header, the lines
    // (written by a few threads at their offsets) and the "/" line
    const int fd = open(filename, O_RDWR | O_CREAT | O_TRUNC, 0666);
    if (fd < 0)
        throw HpglError{HPGL_E_INVALID, std::string("open_file_checked: Can't open file '") + filename + "'."};
    struct FdCloser {
        int fd;
        ~FdCloser() {
            if (fd >= 0) close(fd);
        }
    } closer{fd};
    const std::string head = std::string(format == 1 ? "HPGL saved GSLIB file\n1\n" : "") + name + "\n";
    const std::string tail = format == 0 ? "/\n" : "";
    write_file(fd, head.data(), (long long)head.size(), 0);
    write_file(fd, h, body, (long long)head.size());
    write_file(fd, tail.data(), (long long)tail.size(), (long long)head.size() + body);
    close(fd);  // inside the timing: closing a freshly written file can take a while
    closer.fd = -1;
    tm.ms_file = ms_since(t0);
    tm.bytes = body;
    tm.tokens = size;
    tm.ms_total = ms_since(t_start);
    g_last_timing = tm;
    if (timing) *timing = tm;
}

}  // namespace hpgl_b200
