// Serving loop: continuous batching of DOp programs (radix-integer IOps
// expanded into digit operations) over device-resident keys.
//
// It replaces the HPU's instruction scheduler + ucore firmware
// (hw/module/instruction_scheduler, fw/ublaze/src/ucore_fw.c:54-130): each
// admitted request is a DOp program over its own register file; every round
// issues all ready linear DOps of all requests in one launch and all ready PBS
// DOps of all requests in one KS+PBS launch (the HPU's PBS batch, here
// spanning requests).  Admission is bounded by a slot pool carved from the
// context's HBM budget; a request enters when its registers and I/O blocks fit,
// and its work joins whatever is already in flight.
//
// DOp words follow the reference's field layouts (fw/ublaze/src/hpu_dop_fmt.h:49-117,
// LSB first): arith {dst:7 src0:7 src1:7 mul_factor:5 opcode:6},
// arith_msg {dst:7 src0:7 msg_mode:1 msg_cst:11 opcode:6},
// mem {rid:7 pad:1 mode:2 slot:16 opcode:6}, pbs {dst:7 src:7 gid:12 opcode:6},
// sync {sid:26 opcode:6}; kind = opcode >> 4 (00 arith, 01 sync, 10 mem,
// 11 pbs) and the arith flag bits IMM 8, MUL 4, SUB 2, ADD 1 (:121-140).
#include <algorithm>
#include <chrono>
#include <deque>
#include <map>
#include <string.h>
#include <thread>
#include <vector>
#include "ctx.h"

using namespace luthe;

namespace {

enum : uint32_t {
    OP_ADD = 0x01, OP_SUB = 0x02, OP_MAC = 0x05, OP_ADDS = 0x09, OP_SUBS = 0x0A, OP_SSUB = 0x0B, OP_MULS = 0x0C,
    OP_SYNC = 0x10, OP_LD = 0x20, OP_ST = 0x21, OP_PBS = 0x30, OP_PBS_ML2 = 0x31, OP_PBS_ML4 = 0x32,
    OP_PBS_ML8 = 0x33, OP_FLUSH = 0x08,  // PBS flush variant: opcode | 0x08
};
enum : uint32_t { MEM_ADDR = 0, MEM_HEAP = 1, MEM_SRC = 2, MEM_DST = 3 };

constexpr uint32_t NREG = 128;  // 7-bit register ids

struct Instr {
    uint8_t kind;      // 0 alu (incl. ld/st copy), 1 pbs, 2 sync
    uint8_t alu_op;    // LweOp or LWE_COPY
    uint8_t mlk;       // pbs outputs
    uint32_t dst, a, b;  // slot offsets within the request
    uint64_t imm;
    uint32_t gid;
    int npred = 0;
    std::vector<int> succ;
    bool done = false;
    std::chrono::steady_clock::time_point t_ready;  // when its last dependency finished
};

using clock_t_ = std::chrono::steady_clock;

struct Request {
    uint64_t id;
    std::vector<Instr> prog;
    uint32_t n_src, n_dst, n_heap, n_slots;
    uint32_t base = 0;         // first device pool slot
    uint32_t hbase = 0;        // first pinned host slot: [src][dst]
    std::vector<int> ready;
    size_t remaining = 0;
    cudaEvent_t retired = nullptr;  // outputs copied back
    clock_t_::time_point t_submit, t_admit, t_done;
};

// request-relative slot layout: [regs 0..127][src][dst][heap]
inline uint32_t reg_slot(uint32_t r) { return r; }

int decode(const uint32_t *dops, uint32_t n, uint32_t n_src, uint32_t n_dst, uint32_t nlut, std::vector<Instr> &out,
           uint32_t &n_heap)
{
    out.clear();
    n_heap = 0;
    for (uint32_t i = 0; i < n; i++) {
        const uint32_t w = dops[i], opc = w >> 26, kind = opc >> 4;
        Instr in{};
        in.mlk = 1;
        if (kind == 0) {  // arith
            const uint32_t dst = w & 0x7F, s0 = (w >> 7) & 0x7F;
            in.kind = 0;
            in.dst = reg_slot(dst);
            in.a = reg_slot(s0);
            if (opc == OP_ADD || opc == OP_SUB || opc == OP_MAC) {
                in.b = reg_slot((w >> 14) & 0x7F);
                in.imm = (w >> 21) & 0x1F;
                in.alu_op = opc == OP_ADD ? LWE_ADD : opc == OP_SUB ? LWE_SUB : LWE_MAC;
            } else if (opc == OP_ADDS || opc == OP_SUBS || opc == OP_SSUB || opc == OP_MULS) {
                if ((w >> 14) & 1) return fail(LUTHE_E_PARAM, "DOp %u: templated immediates are not supported", i);
                in.imm = (w >> 15) & 0x7FF;
                in.alu_op = opc == OP_ADDS ? LWE_ADDS : opc == OP_SUBS ? LWE_SUBS : opc == OP_SSUB ? LWE_SSUB : LWE_MULS;
            } else {
                return fail(LUTHE_E_PARAM, "DOp %u: unknown arith opcode 0x%02x", i, opc);
            }
        } else if (kind == 1) {
            if (opc != OP_SYNC) return fail(LUTHE_E_PARAM, "DOp %u: unknown control opcode 0x%02x", i, opc);
            in.kind = 2;
        } else if (kind == 2) {  // LD / ST
            const uint32_t rid = w & 0x7F, mode = (w >> 8) & 3, slot = (w >> 10) & 0xFFFF;
            uint32_t mem;
            if (mode == MEM_SRC) {
                if (slot >= n_src) return fail(LUTHE_E_PARAM, "DOp %u: source block %u >= %u", i, slot, n_src);
                mem = NREG + slot;
            } else if (mode == MEM_DST) {
                if (slot >= n_dst) return fail(LUTHE_E_PARAM, "DOp %u: destination block %u >= %u", i, slot, n_dst);
                mem = NREG + n_src + slot;
            } else if (mode == MEM_HEAP) {
                if (slot >= 1024) return fail(LUTHE_E_PARAM, "DOp %u: heap slot %u too large", i, slot);
                if (slot + 1 > n_heap) n_heap = slot + 1;
                mem = NREG + n_src + n_dst + slot;
            } else {
                return fail(LUTHE_E_PARAM, "DOp %u: absolute memory addressing is not supported", i);
            }
            in.kind = 0;
            in.alu_op = LWE_COPY;
            if (opc == OP_LD) {
                in.dst = reg_slot(rid);
                in.a = mem;
            } else if (opc == OP_ST) {
                in.dst = mem;
                in.a = reg_slot(rid);
            } else {
                return fail(LUTHE_E_PARAM, "DOp %u: unknown memory opcode 0x%02x", i, opc);
            }
        } else {  // PBS
            const uint32_t base = opc & ~OP_FLUSH;
            if (base < OP_PBS || base > OP_PBS_ML8) return fail(LUTHE_E_PARAM, "DOp %u: unknown PBS opcode 0x%02x", i, opc);
            in.kind = 1;
            in.mlk = (uint8_t)(1u << (base - OP_PBS));
            in.dst = reg_slot(w & 0x7F);
            in.a = reg_slot((w >> 7) & 0x7F);
            in.gid = (w >> 14) & 0xFFF;
            if (in.gid >= nlut) return fail(LUTHE_E_PARAM, "DOp %u: LUT %u not uploaded (%u LUTs)", i, in.gid, nlut);
            if (in.dst % in.mlk || in.dst + in.mlk > NREG)
                return fail(LUTHE_E_PARAM, "DOp %u: many-LUT destination R%u not aligned to %u", i, in.dst, in.mlk);
        }
        out.push_back(in);
    }
    return LUTHE_OK;
}

// Dependencies: read-after-write, write-after-write and write-after-read on
// request slots; SYNC orders everything before it before everything after it.
void build_dag(Request &r)
{
    const uint32_t nslot = r.n_slots;
    std::vector<int> last_w(nslot, -1);
    std::vector<std::vector<int>> readers(nslot);
    int last_sync = -1;
    std::vector<int> since_sync;
    auto edge = [&](int from, int to) {
        if (from < 0 || from == to) return;
        r.prog[from].succ.push_back(to);
        r.prog[to].npred++;
    };
    for (int i = 0; i < (int)r.prog.size(); i++) {
        Instr &in = r.prog[i];
        if (in.kind == 2) {
            for (int j : since_sync) edge(j, i);
            since_sync.clear();
            last_sync = i;
            continue;
        }
        edge(last_sync, i);
        since_sync.push_back(i);
        std::vector<uint32_t> srcs{in.a};
        if (in.kind == 0 && (in.alu_op == LWE_ADD || in.alu_op == LWE_SUB || in.alu_op == LWE_MAC)) srcs.push_back(in.b);
        for (uint32_t s : srcs) edge(last_w[s], i);
        for (uint32_t d = in.dst; d < in.dst + (in.kind == 1 ? in.mlk : 1u); d++) {
            edge(last_w[d], i);
            for (int rd : readers[d]) edge(rd, i);
            readers[d].clear();
            last_w[d] = i;
        }
        for (uint32_t s : srcs) readers[s].push_back(i);
    }
    // de-duplicate successor lists so counts match
    for (auto &in : r.prog) in.npred = 0;
    for (auto &in : r.prog) {
        std::vector<int> u;
        for (int s : in.succ)
            if (u.empty() || std::find(u.begin(), u.end(), s) == u.end()) u.push_back(s);
        in.succ.swap(u);
    }
    for (auto &in : r.prog)
        for (int s : in.succ) r.prog[s].npred++;
    r.ready.clear();
    const auto now = clock_t_::now();
    for (int i = 0; i < (int)r.prog.size(); i++)
        if (r.prog[i].npred == 0) {
            r.prog[i].t_ready = now;
            r.ready.push_back(i);
        }
    r.remaining = r.prog.size();
}

// First-fit allocator over slot ranges (device pool and pinned host staging).
struct SlotPool {
    std::vector<std::pair<uint32_t, uint32_t>> free_list;  // (start, len), sorted
    void init(uint32_t n) { free_list.assign(1, {0, n}); }
    bool alloc(uint32_t len, uint32_t &start)
    {
        for (size_t i = 0; i < free_list.size(); i++)
            if (free_list[i].second >= len) {
                start = free_list[i].first;
                free_list[i].first += len;
                free_list[i].second -= len;
                if (free_list[i].second == 0) free_list.erase(free_list.begin() + i);
                return true;
            }
        return false;
    }
    void release(uint32_t start, uint32_t len)
    {
        if (!len) return;
        auto it = free_list.begin();
        while (it != free_list.end() && it->first < start) ++it;
        auto ins = free_list.insert(it, {start, len});  // may reallocate: take begin() after it
        size_t i = ins - free_list.begin();
        if (i + 1 < free_list.size() && free_list[i].first + free_list[i].second == free_list[i + 1].first) {
            free_list[i].second += free_list[i + 1].second;
            free_list.erase(free_list.begin() + i + 1);
        }
        if (i > 0 && free_list[i - 1].first + free_list[i - 1].second == free_list[i].first) {
            free_list[i - 1].second += free_list[i].second;
            free_list.erase(free_list.begin() + i);
        }
    }
};

// One PBS lane: a stream with its own KS scratch and index arrays, so that
// batches issued at different times run concurrently on the GPU.
struct Lane {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    uint32_t *d_l2n = nullptr;   // [max_pbs][n+1]
    uint32_t *d_idx = nullptr;   // [3][max_pbs]: src, dst, gid
    uint32_t *d_part = nullptr;  // split-K partial sums of this lane's small key switches (kept zero)
    uint32_t *h_idx = nullptr;   // pinned staging of d_idx
    std::vector<std::pair<Request *, int>> ops;
    bool busy = false;
};

// Small batches run in the latency forms on a few SMs each for about 7 ms
// whatever their size: enough lanes let many of them share the 148 SMs.
constexpr int LANES = 16;

}  // namespace

struct luthe_server {
    luthe_ctx *ctx = nullptr;
    uint64_t *d_pool = nullptr;
    uint32_t nslots = 0;
    SlotPool dev, host;
    uint64_t *h_pool = nullptr;  // pinned staging, same slot size
    uint32_t nhost = 0;
    std::deque<Request *> pending;
    std::vector<Request *> active, retiring;
    std::map<uint64_t, Request *> done;
    uint64_t next_id = 1;
    cudaStream_t alu_stream = nullptr;
    cudaEvent_t alu_done = nullptr;
    Lane lanes[LANES];
    AluOp *d_ops = nullptr, *h_ops = nullptr;  // pinned ring of ALU descriptors
    uint32_t ops_cap = 0, ops_head = 0;
    uint32_t max_pbs = 4096;
    uint64_t rounds = 0, pbs_done = 0, alu_done_n = 0, launches = 0;
    // batching window (luthe_server_set_batching): 0 = off
    uint32_t fill = 0;
    double window_s = 0;
    uint64_t held = 0;  // rounds in which ready PBS were held back
};

namespace {

int check_err(luthe_ctx *c)
{
    uint32_t e = 0;
    CUDA_TRY(cudaMemcpy(&e, c->d_err, 4, cudaMemcpyDeviceToHost));
    if (e) return fail(LUTHE_E_TIMEOUT, "blind rotation: bounded wait for a BSK slab ran out");
    return LUTHE_OK;
}

void finish(Request *r, int i)
{
    r->prog[i].done = true;
    r->remaining--;
    for (int j : r->prog[i].succ)
        if (--r->prog[j].npred == 0) {
            r->prog[j].t_ready = clock_t_::now();
            r->ready.push_back(j);
        }
}

}  // namespace

extern "C" int luthe_server_create(luthe_ctx *c, uint64_t pool_bytes, uint32_t max_pbs, luthe_server **out)
{
    if (!c || !out) return fail(LUTHE_E_PARAM, "null argument");
    *out = nullptr;
    int r = need_keys(c);
    if (r) return r;
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t slot_bytes = (size_t)(c->p.poly_size + 1) * 8;
    const uint64_t nslots = pool_bytes / slot_bytes;
    if (nslots < 2 * NREG || nslots > 0xFFFFFFFFull)
        return fail(LUTHE_E_PARAM, "pool of %llu slots is out of range", (unsigned long long)nslots);
    luthe_server *s = new luthe_server();
    s->ctx = c;
    s->nslots = (uint32_t)nslots;
    s->max_pbs = max_pbs ? max_pbs : 4096;
    s->nhost = (uint32_t)std::min<uint64_t>(nslots, 65536);
    s->ops_cap = 1u << 16;
    const size_t n1 = c->p.lwe_dim + 1;
    bool ok = !dalloc(c, (void **)&s->d_pool, nslots * slot_bytes) &&
              !dalloc(c, (void **)&s->d_ops, (size_t)s->ops_cap * sizeof(AluOp)) &&
              cudaMallocHost((void **)&s->h_pool, (size_t)s->nhost * slot_bytes) == cudaSuccess &&
              cudaMallocHost((void **)&s->h_ops, (size_t)s->ops_cap * sizeof(AluOp)) == cudaSuccess &&
              cudaStreamCreateWithFlags(&s->alu_stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&s->alu_done, cudaEventDisableTiming) == cudaSuccess;
    for (int l = 0; ok && l < LANES; l++) {
        Lane &ln = s->lanes[l];
        ok = !dalloc(c, (void **)&ln.d_l2n, (size_t)s->max_pbs * n1 * 4) &&
             !dalloc(c, (void **)&ln.d_part, (size_t)KS_BM * c->xpad * 4) &&
             cudaMemset(ln.d_part, 0, (size_t)KS_BM * c->xpad * 4) == cudaSuccess &&
             !dalloc(c, (void **)&ln.d_idx, (size_t)s->max_pbs * 3 * 4) &&
             cudaMallocHost((void **)&ln.h_idx, (size_t)s->max_pbs * 3 * 4) == cudaSuccess &&
             cudaStreamCreateWithFlags(&ln.stream, cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&ln.done, cudaEventDisableTiming) == cudaSuccess;
    }
    if (!ok) {
        luthe_server_destroy(s);
        return fail(LUTHE_E_BUDGET, "server resources could not be allocated (%s)", g_err);
    }
    s->dev.init(s->nslots);
    s->host.init(s->nhost);
    *out = s;
    return LUTHE_OK;
}

extern "C" void luthe_server_destroy(luthe_server *s)
{
    if (!s) return;
    luthe_ctx *c = s->ctx;
    cudaSetDevice(c->device);
    const size_t n1 = c->p.lwe_dim + 1;
    cudaDeviceSynchronize();
    for (Lane &ln : s->lanes) {
        if (ln.stream) cudaStreamDestroy(ln.stream);
        if (ln.done) cudaEventDestroy(ln.done);
        if (ln.h_idx) cudaFreeHost(ln.h_idx);
        dfree(c, ln.d_l2n, ln.d_l2n ? (size_t)s->max_pbs * n1 * 4 : 0);
        dfree(c, ln.d_idx, ln.d_idx ? (size_t)s->max_pbs * 3 * 4 : 0);
        dfree(c, ln.d_part, ln.d_part ? (size_t)KS_BM * c->xpad * 4 : 0);
    }
    if (s->alu_stream) cudaStreamDestroy(s->alu_stream);
    if (s->alu_done) cudaEventDestroy(s->alu_done);
    if (s->h_pool) cudaFreeHost(s->h_pool);
    if (s->h_ops) cudaFreeHost(s->h_ops);
    dfree(c, s->d_pool, s->d_pool ? (size_t)s->nslots * (c->p.poly_size + 1) * 8 : 0);
    dfree(c, s->d_ops, s->d_ops ? (size_t)s->ops_cap * sizeof(AluOp) : 0);
    auto drop = [](Request *r) {
        if (r->retired) cudaEventDestroy(r->retired);
        delete r;
    };
    for (auto *r : s->pending) drop(r);
    for (auto *r : s->active) drop(r);
    for (auto *r : s->retiring) drop(r);
    for (auto &kv : s->done) drop(kv.second);
    delete s;
}

extern "C" int luthe_server_submit(luthe_server *s, const uint32_t *dops, uint32_t n_dops, const uint64_t *h_src,
                                   uint32_t n_src, uint32_t n_dst, uint64_t *id)
{
    if (!s || !dops || !id || (n_src && !h_src)) return fail(LUTHE_E_PARAM, "null argument");
    if (n_src > 0xFFFF || n_dst > 0xFFFF) return fail(LUTHE_E_PARAM, "too many I/O blocks");
    Request *r = new Request();
    int rc = decode(dops, n_dops, n_src, n_dst, s->ctx->nlut, r->prog, r->n_heap);
    if (rc) {
        delete r;
        return rc;
    }
    r->n_src = n_src;
    r->n_dst = n_dst;
    r->n_slots = NREG + n_src + n_dst + r->n_heap;
    if (r->n_slots > s->nslots) {
        delete r;
        return fail(LUTHE_E_BUDGET, "request needs %u slots, the pool has %u", r->n_slots, s->nslots);
    }
    if (!s->host.alloc(n_src + n_dst, r->hbase)) {
        delete r;
        return fail(LUTHE_E_BUDGET, "pinned staging full: retire finished requests first");
    }
    const size_t w = s->ctx->p.poly_size + 1;
    memcpy(s->h_pool + (size_t)r->hbase * w, h_src, (size_t)n_src * w * 8);
    r->id = s->next_id++;
    r->t_submit = clock_t_::now();
    s->pending.push_back(r);
    *id = r->id;
    return LUTHE_OK;
}

// One pass of the asynchronous scheduler: harvest finished PBS lanes and
// retirements, admit, issue ready linear DOps, issue ready PBS on idle lanes.
extern "C" int luthe_server_step(luthe_server *s, uint32_t *n_completed, uint32_t *n_active, uint32_t *n_pending)
{
    if (!s) return fail(LUTHE_E_PARAM, "null server");
    luthe_ctx *c = s->ctx;
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t w = c->p.poly_size + 1;
    const uint32_t n = c->p.lwe_dim;
    uint32_t completed = 0;
    bool progress = false;

    // PBS lanes whose batch finished: their DOps are done
    for (Lane &ln : s->lanes) {
        if (!ln.busy) continue;
        cudaError_t q = cudaEventQuery(ln.done);
        if (q == cudaErrorNotReady) continue;
        CUDA_TRY(q);
        for (auto &p : ln.ops) finish(p.first, p.second);
        ln.ops.clear();
        ln.busy = false;
        progress = true;
        int r = check_err(c);
        if (r) return r;
    }
    // requests whose outputs reached the pinned staging
    for (size_t i = 0; i < s->retiring.size();) {
        Request *r = s->retiring[i];
        cudaError_t q = cudaEventQuery(r->retired);
        if (q == cudaErrorNotReady) {
            i++;
            continue;
        }
        CUDA_TRY(q);
        r->t_done = clock_t_::now();
        cudaEventDestroy(r->retired);
        r->retired = nullptr;
        s->dev.release(r->base, r->n_slots);
        s->done[r->id] = r;
        s->retiring.erase(s->retiring.begin() + i);
        completed++;
        progress = true;
    }
    // admission: FIFO while the device pool has room
    while (!s->pending.empty()) {
        Request *r = s->pending.front();
        uint32_t base;
        if (!s->dev.alloc(r->n_slots, base)) break;
        s->pending.pop_front();
        r->base = base;
        r->t_admit = clock_t_::now();
        if (r->n_src)
            CUDA_TRY(cudaMemcpyAsync(s->d_pool + (size_t)(base + NREG) * w, s->h_pool + (size_t)r->hbase * w,
                                     (size_t)r->n_src * w * 8, cudaMemcpyHostToDevice, s->alu_stream));
        build_dag(*r);
        s->active.push_back(r);
        progress = true;
    }
    // linear DOps, LD/ST copies and SYNCs, in waves on the ALU stream; they are
    // stream-ordered, and PBS lanes wait on the ALU stream before reading
    bool alu_issued = false;
    for (;;) {
        std::vector<AluOp> ops;
        std::vector<std::pair<Request *, int>> issued;
        for (Request *r : s->active) {
            std::vector<int> keep;
            for (int i : r->ready) {
                Instr &in = r->prog[i];
                if (in.kind == 1 || (in.kind == 0 && ops.size() >= s->ops_cap / 2)) {
                    keep.push_back(i);
                    continue;
                }
                if (in.kind == 0) ops.push_back(AluOp{in.alu_op, r->base + in.dst, r->base + in.a, r->base + in.b, in.imm});
                issued.push_back({r, i});
            }
            r->ready.swap(keep);
        }
        if (issued.empty()) break;
        if (!ops.empty()) {
            // descriptors go through a pinned ring; before the ring wraps, the
            // copies still reading its start must have finished
            uint32_t head = s->ops_head;
            if (head + ops.size() > s->ops_cap) {
                CUDA_TRY(cudaStreamSynchronize(s->alu_stream));
                head = 0;
            }
            memcpy(s->h_ops + head, ops.data(), ops.size() * sizeof(AluOp));
            CUDA_TRY(cudaMemcpyAsync(s->d_ops + head, s->h_ops + head, ops.size() * sizeof(AluOp),
                                     cudaMemcpyHostToDevice, s->alu_stream));
            CUDA_TRY(launch_alu_batch(s->d_ops + head, s->d_pool, (uint32_t)ops.size(), c->p.poly_size,
                                      s->alu_stream));
            s->ops_head = head + (uint32_t)ops.size();
            s->launches++;
            s->alu_done_n += ops.size();
            alu_issued = true;
        }
        for (auto &p : issued) finish(p.first, p.second);
        progress = true;
    }
    if (alu_issued) CUDA_TRY(cudaEventRecord(s->alu_done, s->alu_stream));
    // finished requests: copy outputs back on the ALU stream
    std::vector<Request *> still;
    for (Request *r : s->active) {
        if (r->remaining) {
            still.push_back(r);
            continue;
        }
        if (r->n_dst)
            CUDA_TRY(cudaMemcpyAsync(s->h_pool + (size_t)(r->hbase + r->n_src) * w,
                                     s->d_pool + (size_t)(r->base + NREG + r->n_src) * w, (size_t)r->n_dst * w * 8,
                                     cudaMemcpyDeviceToHost, s->alu_stream));
        CUDA_TRY(cudaEventCreateWithFlags(&r->retired, cudaEventDisableTiming));
        CUDA_TRY(cudaEventRecord(r->retired, s->alu_stream));
        s->retiring.push_back(r);
        progress = true;
    }
    s->active.swap(still);
    // ready PBS on idle lanes (one many-LUT factor per batch)
    for (Lane &ln : s->lanes) {
        if (ln.busy) continue;
        uint32_t mlk = 0, B = 0, nready = 0;
        clock_t_::time_point oldest = clock_t_::time_point::max();
        for (Request *r : s->active)
            for (int i : r->ready)
                if (r->prog[i].kind == 1) {
                    if (!mlk) mlk = r->prog[i].mlk;
                    if (r->prog[i].mlk == mlk) {
                        nready++;
                        oldest = std::min(oldest, r->prog[i].t_ready);
                    }
                }
        if (!mlk) break;
        if (s->window_s > 0) {
            // the HPU's batch policy: a batch leaves when full or when its
            // oldest entry has waited the timeout; while the GPU is idle there
            // is nothing to wait for
            bool any_busy = false;
            for (const Lane &o : s->lanes) any_busy |= o.busy;
            const uint32_t fill = s->fill ? s->fill : 2u * (uint32_t)c->nsm;
            const double waited = std::chrono::duration<double>(clock_t_::now() - oldest).count();
            if (any_busy && nready < fill && waited < s->window_s) {
                s->held++;
                break;
            }
        }
        for (Request *r : s->active) {
            std::vector<int> keep;
            for (int i : r->ready) {
                Instr &in = r->prog[i];
                if (in.kind == 1 && in.mlk == mlk && B < s->max_pbs) {
                    ln.h_idx[B] = r->base + in.a;
                    ln.h_idx[s->max_pbs + B] = r->base + in.dst;
                    ln.h_idx[2 * s->max_pbs + B] = in.gid;
                    ln.ops.push_back({r, i});
                    B++;
                } else {
                    keep.push_back(i);
                }
            }
            r->ready.swap(keep);
        }
        // Cluster pairs hold two SMs per ciphertext for about 7 ms.  When the
        // ciphertexts already on the GPU and this batch would need more SMs
        // than there are, pairs would queue for SMs; the batch then runs one
        // ciphertext per CTA instead (10.4 ms on one SM: about 40 % more
        // bootstraps per SM-second).
        size_t inflight = 0;
        for (const Lane &o : s->lanes)
            if (o.busy) inflight += o.ops.size();
        BrConfig cfg = c->br;
        if (2 * (inflight + B) > (size_t)c->nsm) cfg.pair_max = 0;
        CUDA_TRY(cudaStreamWaitEvent(ln.stream, s->alu_done, 0));
        CUDA_TRY(cudaMemcpyAsync(ln.d_idx, ln.h_idx, (size_t)s->max_pbs * 3 * 4, cudaMemcpyHostToDevice, ln.stream));
        CUDA_TRY(launch_keyswitch(s->d_pool, c->d_ksk, nullptr, ln.d_l2n, B, n, c->xpad, ln.stream, ln.d_idx, c->p.ks_base_log, c->p.ks_level, c->tie_rule,
                                  ln.d_part));
        CUDA_TRY(launch_blind_rotate(cfg, c->nsm, ln.d_l2n, c->d_luts, ln.d_idx + 2 * s->max_pbs, c->nlut,
                                     c->d_bsk, c->d_tw, s->d_pool, B, n, c->d_err, ln.stream,
                                     ln.d_idx + s->max_pbs, mlk, c->p.pbs_base_log, c->tie_rule));
        CUDA_TRY(cudaEventRecord(ln.done, ln.stream));
        ln.busy = true;
        s->launches += 2;
        s->pbs_done += B;
        s->rounds++;
        progress = true;
    }
    if (!progress) std::this_thread::sleep_for(std::chrono::microseconds(100));  // GPU busy: do not spin
    if (n_completed) *n_completed = completed;
    if (n_active) *n_active = (uint32_t)(s->active.size() + s->retiring.size());
    if (n_pending) *n_pending = (uint32_t)s->pending.size();
    return LUTHE_OK;
}

extern "C" int luthe_server_fetch(luthe_server *s, uint64_t id, uint64_t *h_dst, double *latency_s, double *queue_s)
{
    if (!s) return fail(LUTHE_E_PARAM, "null server");
    auto it = s->done.find(id);
    if (it == s->done.end()) return fail(LUTHE_E_STATE, "request %llu is not complete", (unsigned long long)id);
    Request *r = it->second;
    const size_t w = s->ctx->p.poly_size + 1;
    if (h_dst) memcpy(h_dst, s->h_pool + (size_t)(r->hbase + r->n_src) * w, (size_t)r->n_dst * w * 8);
    if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    if (queue_s) *queue_s = std::chrono::duration<double>(r->t_admit - r->t_submit).count();
    s->host.release(r->hbase, r->n_src + r->n_dst);
    s->done.erase(it);
    delete r;
    return LUTHE_OK;
}

extern "C" int luthe_server_set_batching(luthe_server *s, uint32_t fill, uint32_t window_us)
{
    if (!s) return fail(LUTHE_E_PARAM, "null server");
    if (fill > s->max_pbs) return fail(LUTHE_E_PARAM, "fill %u exceeds the server's batch limit %u", fill, s->max_pbs);
    s->fill = fill;
    s->window_s = window_us * 1e-6;
    return LUTHE_OK;
}

extern "C" int luthe_server_counters(luthe_server *s, uint64_t *rounds, uint64_t *pbs, uint64_t *alu,
                                     uint64_t *launches)
{
    if (!s) return fail(LUTHE_E_PARAM, "null server");
    if (rounds) *rounds = s->rounds;
    if (pbs) *pbs = s->pbs_done;
    if (alu) *alu = s->alu_done_n;
    if (launches) *launches = s->launches;
    return LUTHE_OK;
}
