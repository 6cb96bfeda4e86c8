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
};

using clock_t_ = std::chrono::steady_clock;

struct Request {
    uint64_t id;
    std::vector<Instr> prog;
    uint32_t n_src, n_dst, n_heap, n_slots;
    uint32_t base = 0;         // first pool slot
    std::vector<uint64_t> h_src, h_dst;
    std::vector<int> ready;
    size_t remaining = 0;
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
    for (int i = 0; i < (int)r.prog.size(); i++)
        if (r.prog[i].npred == 0) r.ready.push_back(i);
    r.remaining = r.prog.size();
}

}  // namespace

struct luthe_server {
    luthe_ctx *ctx = nullptr;
    uint64_t *d_pool = nullptr;
    uint32_t nslots = 0;
    std::vector<std::pair<uint32_t, uint32_t>> free_list;  // (start, len), sorted
    std::deque<Request *> pending;
    std::vector<Request *> active;
    std::map<uint64_t, Request *> done;
    uint64_t next_id = 1;
    cudaStream_t stream = nullptr;
    AluOp *d_ops = nullptr;
    uint32_t ops_cap = 0;
    uint32_t *d_idx = nullptr;  // [src | dst | gid] of a PBS batch
    uint32_t idx_cap = 0;
    uint32_t max_pbs = 4096;
    uint64_t rounds = 0, pbs_done = 0, alu_done = 0, launches = 0;
};

static bool pool_alloc(luthe_server *s, uint32_t len, uint32_t &start)
{
    for (size_t i = 0; i < s->free_list.size(); i++)
        if (s->free_list[i].second >= len) {
            start = s->free_list[i].first;
            s->free_list[i].first += len;
            s->free_list[i].second -= len;
            if (s->free_list[i].second == 0) s->free_list.erase(s->free_list.begin() + i);
            return true;
        }
    return false;
}
static void pool_free(luthe_server *s, uint32_t start, uint32_t len)
{
    auto it = s->free_list.begin();
    while (it != s->free_list.end() && it->first < start) ++it;
    it = s->free_list.insert(it, {start, len});
    // merge with neighbours
    size_t i = it - s->free_list.begin();
    if (i + 1 < s->free_list.size() && s->free_list[i].first + s->free_list[i].second == s->free_list[i + 1].first) {
        s->free_list[i].second += s->free_list[i + 1].second;
        s->free_list.erase(s->free_list.begin() + i + 1);
    }
    if (i > 0 && s->free_list[i - 1].first + s->free_list[i - 1].second == s->free_list[i].first) {
        s->free_list[i - 1].second += s->free_list[i].second;
        s->free_list.erase(s->free_list.begin() + i);
    }
}

extern "C" int luthe_server_create(luthe_ctx *c, uint64_t pool_bytes, uint32_t max_pbs, luthe_server **out)
{
    if (!c || !out) return fail(LUTHE_E_PARAM, "null argument");
    *out = nullptr;
    int r = need_keys(c);
    if (r) return r;
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t slot_bytes = (size_t)(c->p.poly_size + 1) * 8;
    const uint64_t nslots = pool_bytes / slot_bytes;
    if (nslots < 2 * NREG || nslots > 0xFFFFFFFFull) return fail(LUTHE_E_PARAM, "pool of %llu slots is out of range",
                                                                  (unsigned long long)nslots);
    luthe_server *s = new luthe_server();
    s->ctx = c;
    s->nslots = (uint32_t)nslots;
    s->max_pbs = max_pbs ? max_pbs : 4096;
    if ((r = dalloc(c, (void **)&s->d_pool, nslots * slot_bytes)) || (r = ensure_scratch(c, s->max_pbs)) ||
        (r = dalloc(c, (void **)&s->d_idx, (size_t)s->max_pbs * 3 * 4))) {
        luthe_server_destroy(s);
        return r;
    }
    s->idx_cap = s->max_pbs;
    s->free_list.push_back({0, s->nslots});
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
        luthe_server_destroy(s);
        return fail(LUTHE_E_CUDA, "stream creation failed");
    }
    *out = s;
    return LUTHE_OK;
}

extern "C" void luthe_server_destroy(luthe_server *s)
{
    if (!s) return;
    luthe_ctx *c = s->ctx;
    cudaSetDevice(c->device);
    if (s->stream) {
        cudaStreamSynchronize(s->stream);
        cudaStreamDestroy(s->stream);
    }
    dfree(c, s->d_pool, (size_t)s->nslots * (c->p.poly_size + 1) * 8);
    dfree(c, s->d_ops, (size_t)s->ops_cap * sizeof(AluOp));
    dfree(c, s->d_idx, (size_t)s->idx_cap * 3 * 4);
    for (auto *r : s->pending) delete r;
    for (auto *r : s->active) delete r;
    for (auto &kv : s->done) delete kv.second;
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
    const size_t w = s->ctx->p.poly_size + 1;
    r->h_src.assign(h_src, h_src + (size_t)n_src * w);
    r->h_dst.assign((size_t)n_dst * w, 0);
    r->id = s->next_id++;
    r->t_submit = clock_t_::now();
    s->pending.push_back(r);
    *id = r->id;
    return LUTHE_OK;
}

// one scheduling round: admit, linear waves, one PBS batch, retire
extern "C" int luthe_server_step(luthe_server *s, uint32_t *n_completed, uint32_t *n_active, uint32_t *n_pending)
{
    if (!s) return fail(LUTHE_E_PARAM, "null server");
    luthe_ctx *c = s->ctx;
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t w = c->p.poly_size + 1;
    const uint32_t n = c->p.lwe_dim;
    uint32_t completed = 0;

    // admission: FIFO while the pool has room
    while (!s->pending.empty()) {
        Request *r = s->pending.front();
        uint32_t base;
        if (!pool_alloc(s, r->n_slots, base)) break;
        s->pending.pop_front();
        r->base = base;
        r->t_admit = clock_t_::now();
        if (r->n_src)
            CUDA_TRY(cudaMemcpyAsync(s->d_pool + (size_t)(base + NREG) * w, r->h_src.data(), r->h_src.size() * 8,
                                     cudaMemcpyHostToDevice, s->stream));
        build_dag(*r);
        s->active.push_back(r);
    }

    auto finish = [&](Request *r, int i) {
        r->prog[i].done = true;
        r->remaining--;
        for (int j : r->prog[i].succ)
            if (--r->prog[j].npred == 0) r->ready.push_back(j);
    };

    // linear DOps, LD/ST copies and SYNCs: waves until none is ready
    for (;;) {
        std::vector<AluOp> ops;
        std::vector<std::pair<Request *, int>> issued;
        for (Request *r : s->active) {
            std::vector<int> keep;
            for (int i : r->ready) {
                Instr &in = r->prog[i];
                if (in.kind == 1) {
                    keep.push_back(i);
                } else if (in.kind == 2) {
                    issued.push_back({r, i});
                } else {
                    ops.push_back(AluOp{in.alu_op, r->base + in.dst, r->base + in.a, r->base + in.b, in.imm});
                    issued.push_back({r, i});
                }
            }
            r->ready.swap(keep);
        }
        if (issued.empty()) break;
        if (!ops.empty()) {
            if (ops.size() > s->ops_cap) {
                dfree(c, s->d_ops, (size_t)s->ops_cap * sizeof(AluOp));
                s->d_ops = nullptr;
                s->ops_cap = 0;
                uint32_t cap = (uint32_t)ops.size() * 2;
                int r = dalloc(c, (void **)&s->d_ops, (size_t)cap * sizeof(AluOp));
                if (r) return r;
                s->ops_cap = cap;
            }
            CUDA_TRY(cudaMemcpyAsync(s->d_ops, ops.data(), ops.size() * sizeof(AluOp), cudaMemcpyHostToDevice,
                                     s->stream));
            CUDA_TRY(launch_alu_batch(s->d_ops, s->d_pool, (uint32_t)ops.size(), c->p.poly_size, s->stream));
            s->launches++;
            s->alu_done += ops.size();
        }
        for (auto &p : issued) finish(p.first, p.second);
    }

    // one PBS batch across requests (per many-LUT factor)
    for (uint32_t mlk : {1u, 2u, 4u, 8u}) {
        std::vector<uint32_t> src, dst, gid;
        std::vector<std::pair<Request *, int>> issued;
        for (Request *r : s->active) {
            std::vector<int> keep;
            for (int i : r->ready) {
                Instr &in = r->prog[i];
                if (in.kind == 1 && in.mlk == mlk && src.size() < s->max_pbs) {
                    src.push_back(r->base + in.a);
                    dst.push_back(r->base + in.dst);
                    gid.push_back(in.gid);
                    issued.push_back({r, i});
                } else {
                    keep.push_back(i);
                }
            }
            r->ready.swap(keep);
        }
        if (issued.empty()) continue;
        const uint32_t B = (uint32_t)src.size();
        std::vector<uint32_t> idx(3 * (size_t)B);
        memcpy(idx.data(), src.data(), B * 4);
        memcpy(idx.data() + B, dst.data(), B * 4);
        memcpy(idx.data() + 2 * (size_t)B, gid.data(), B * 4);
        CUDA_TRY(cudaMemcpyAsync(s->d_idx, idx.data(), idx.size() * 4, cudaMemcpyHostToDevice, s->stream));
        CUDA_TRY(launch_keyswitch(s->d_pool, c->d_ksk, nullptr, c->d_lwe2N, B, n, c->xpad, s->stream, s->d_idx));
        CUDA_TRY(launch_blind_rotate(c->br, c->nsm, c->d_lwe2N, c->d_luts, s->d_idx + 2 * (size_t)B, c->nlut, c->d_bsk,
                                     c->d_tw, s->d_pool, B, n, c->d_err, s->stream, s->d_idx + B, mlk));
        s->launches += 2;
        s->pbs_done += B;
        for (auto &p : issued) finish(p.first, p.second);
    }
    s->rounds++;

    CUDA_TRY(cudaStreamSynchronize(s->stream));
    uint32_t e = 0;
    CUDA_TRY(cudaMemcpy(&e, c->d_err, 4, cudaMemcpyDeviceToHost));
    if (e) return fail(LUTHE_E_TIMEOUT, "blind rotation: bounded wait for a BSK slab ran out");

    // retire finished requests
    std::vector<Request *> still;
    for (Request *r : s->active) {
        if (r->remaining) {
            still.push_back(r);
            continue;
        }
        if (r->n_dst)
            CUDA_TRY(cudaMemcpy(r->h_dst.data(), s->d_pool + (size_t)(r->base + NREG + r->n_src) * w,
                                r->h_dst.size() * 8, cudaMemcpyDeviceToHost));
        r->t_done = clock_t_::now();
        pool_free(s, r->base, r->n_slots);
        r->h_src.clear();
        r->h_src.shrink_to_fit();
        r->prog.clear();
        r->prog.shrink_to_fit();
        s->done[r->id] = r;
        completed++;
    }
    s->active.swap(still);
    if (n_completed) *n_completed = completed;
    if (n_active) *n_active = (uint32_t)s->active.size();
    if (n_pending) *n_pending = (uint32_t)s->pending.size();
    return LUTHE_OK;
}

extern "C" int luthe_server_fetch(luthe_server *s, uint64_t id, uint64_t *h_dst, double *latency_s, double *queue_s)
{
    if (!s) return fail(LUTHE_E_PARAM, "null server");
    auto it = s->done.find(id);
    if (it == s->done.end()) return fail(LUTHE_E_STATE, "request %llu is not complete", (unsigned long long)id);
    Request *r = it->second;
    if (h_dst) memcpy(h_dst, r->h_dst.data(), r->h_dst.size() * 8);
    if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    if (queue_s) *queue_s = std::chrono::duration<double>(r->t_admit - r->t_submit).count();
    s->done.erase(it);
    delete r;
    return LUTHE_OK;
}

extern "C" int luthe_server_counters(luthe_server *s, uint64_t *rounds, uint64_t *pbs, uint64_t *alu,
                                     uint64_t *launches)
{
    if (!s) return fail(LUTHE_E_PARAM, "null server");
    if (rounds) *rounds = s->rounds;
    if (pbs) *pbs = s->pbs_done;
    if (alu) *alu = s->alu_done;
    if (launches) *launches = s->launches;
    return LUTHE_OK;
}
