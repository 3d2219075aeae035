// batch.cu -- many shards proven concurrently on one GPU (batched and served modes).
//
// A zkVM run yields many shards of uneven size; each shard is an independent
// fold-step chain (own transcript, own accumulator: crates/neo-fold/src/shard.rs:1725-2283).
// The engine runs W worker threads, each with its own context (CUDA stream).
// Requests wait in one FIFO queue; an idle worker takes the request at its
// head once its device footprint fits the HBM budget (free memory when the
// engine was last idle, minus the footprints of running requests and a
// margin) and proves it to completion.  Host-side Fiat-Shamir work of
// different shards thus runs in parallel on W threads and their kernels
// overlap on the device.  A step of one request is a single-threaded chain
// (transcript, then kernels, then transcript), so a worker that interleaved
// several requests would gain no throughput and only delay each of them:
// run to completion keeps the latency of a request close to its own service
// time plus its queueing.  Worker threads allocate shard buffers from the
// device's memory pool, ordered on their own stream: cudaFree waits for the
// whole device, so a worker freeing a finished shard would otherwise stall
// every other worker's kernels.
#include "internal.cuh"
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>

typedef struct neo_gpu_shard neo_gpu_shard;
extern "C" int neo_gpu_shard_create(neo_gpu_ctx* ctx, const neo_ccs_desc* ccs, uint32_t m_in, uint32_t k_rho,
                                    const char* app_label, neo_gpu_shard** out);
extern "C" int neo_gpu_shard_create_mem(neo_gpu_ctx* ctx, const neo_ccs_desc* ccs, uint32_t m_in, uint32_t k_rho,
                                        const char* app_label, const neo_mem_desc* mem, neo_gpu_shard** out);
extern "C" int neo_gpu_shard_fold_step(neo_gpu_shard* sh, const uint64_t* z, uint64_t* proof, uint64_t proof_cap,
                                       uint64_t* proof_len);
extern "C" int neo_gpu_shard_transcript_state(const neo_gpu_shard* sh, uint64_t* st8);
extern "C" int neo_gpu_shard_destroy(neo_gpu_shard* sh);

namespace {

using bclock = std::chrono::steady_clock;

// Owned copy of a CCS description (the caller's arrays may go away).
struct CcsCopy {
    neo_ccs_desc d{};
    std::vector<uint8_t> is_identity;
    std::vector<uint64_t> col_ptr, nnz_off, vals, f_coeff;
    std::vector<uint32_t> row_idx, f_exps;
    explicit CcsCopy(const neo_ccs_desc* s) {
        is_identity.assign(s->is_identity, s->is_identity + s->t);
        col_ptr.assign(s->col_ptr, s->col_ptr + (size_t)s->t * (s->m + 1));
        nnz_off.assign(s->nnz_off, s->nnz_off + s->t + 1);
        const uint64_t nnz = nnz_off.back();
        row_idx.assign(s->row_idx, s->row_idx + nnz);
        vals.assign(s->vals, s->vals + nnz);
        f_coeff.assign(s->f_coeff, s->f_coeff + s->n_terms);
        f_exps.assign(s->f_exps, s->f_exps + (size_t)s->n_terms * s->t);
        d = *s;
        d.is_identity = is_identity.data();
        d.col_ptr = col_ptr.data();
        d.nnz_off = nnz_off.data();
        d.row_idx = row_idx.data();
        d.vals = vals.data();
        d.f_coeff = f_coeff.data();
        d.f_exps = f_exps.data();
    }
};

// Owned copy of a memory description (tables and initial memories).
struct MemCopy {
    neo_mem_desc d{};
    std::vector<neo_mem_instance> shout, twist;
    std::vector<std::vector<uint64_t>> bufs;
    explicit MemCopy(const neo_mem_desc* s) {
        d = *s;
        auto own = [&](const uint64_t* p, uint64_t n) -> const uint64_t* {
            if (!p || !n) return nullptr;
            bufs.emplace_back(p, p + n);
            return bufs.back().data();
        };
        bufs.reserve(3 * (s->n_shout + s->n_twist) + 1);
        for (uint32_t i = 0; i < s->n_shout; i++) {
            neo_mem_instance m = s->shout[i];
            m.table = own(m.table, m.table_len);
            shout.push_back(m);
        }
        for (uint32_t i = 0; i < s->n_twist; i++) {
            neo_mem_instance m = s->twist[i];
            m.init_addr = own(m.init_addr, m.n_init);
            m.init_val = own(m.init_val, m.n_init);
            twist.push_back(m);
        }
        d.shout = shout.data();
        d.twist = twist.data();
    }
};

struct Job {
    uint64_t id = 0;
    std::unique_ptr<CcsCopy> ccs;
    std::unique_ptr<MemCopy> mem;
    std::vector<uint64_t> z;  // one witness (every step) or n_steps witnesses of m words
    uint32_t n_steps = 0, m_in = 1, k_rho = 12;
    // per step s >= 1 and Twist instance: the MemInit set before step s (empty vector: none given)
    std::vector<std::vector<std::pair<std::vector<uint64_t>, std::vector<uint64_t>>>> inits;
    std::string label;
    uint64_t footprint = 0;
    neo_gpu_shard* shard = nullptr;
    uint32_t steps_done = 0;
    int status = 0;  // 0 pending/running, 1 done, <0 -(error code)
    std::atomic<bool> cancel{false};  // checked by the worker before every fold step
    std::string error;
    bclock::time_point t_submit, t_admit, t_done;
    uint64_t tr_state[8] = {0};
    std::vector<uint64_t> last_proof;
};

struct Worker {
    neo_gpu_ctx* ctx = nullptr;
};

}  // namespace

struct neo_gpu_batch {
    int device = 0;
    std::vector<Worker> workers;
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Job*> pending;                 // submitted, not yet started (FIFO)
    std::vector<std::unique_ptr<Job>> jobs;   // all jobs, by id
    uint64_t reserved = 0;                    // footprints of the running jobs
    uint64_t budget = 0;                      // free HBM when the engine was last idle, minus the margin
    uint64_t reserve_margin = 2ull << 30;     // headroom kept free on the device
    uint64_t unfinished = 0;
    bool stop = false;
    bclock::time_point t0 = bclock::now();
};

// device bytes a shard of size m holds while it is being proven: digit planes,
// Pi_CCS tables (K), commitment scratch, fold buffers.
static uint64_t shard_footprint(uint64_t m, uint32_t k_rho) {
    const uint64_t k = 1 + k_rho;
    uint64_t zall = k * 54 * m;
    uint64_t small = 6 * m * 16 * 3 / 2;
    uint64_t nc = k * 54 * (m / 16) * 16 * 3 / 2;
    uint64_t commit_scratch = (uint64_t)k_rho * m * 144 + 64ull * 1024 * 1024;
    uint64_t fold = 54 * m * 4 + 54 * m * 8 + k * 4 * m * 16;
    return zall + small + nc + commit_scratch + fold;
}

// caller holds b->mu: may the head of the queue start now?
static bool head_fits_locked(neo_gpu_batch* b) {
    if (b->pending.empty()) return false;
    if (b->reserved == 0) {
        // idle engine: hand the pool's unused blocks back, refresh the budget; a
        // request larger than it still runs alone
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, b->device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 0;
        b->budget = free_b > b->reserve_margin ? free_b - b->reserve_margin : 0;
        return true;
    }
    return b->reserved + b->pending.front()->footprint <= b->budget;
}

static void finish_job(neo_gpu_batch* b, Job* j, int status, const char* err) {
    if (j->shard) {
        neo_gpu_shard_transcript_state(j->shard, j->tr_state);
        neo_gpu_shard_destroy(j->shard);
        j->shard = nullptr;
    }
    std::lock_guard<std::mutex> lk(b->mu);
    j->status = status;
    if (err) j->error = err;
    j->t_done = bclock::now();
    b->reserved -= std::min(b->reserved, j->footprint);
    b->unfinished--;
    b->cv_work.notify_all();
    b->cv_done.notify_all();
}

// every fold step of one request on this worker's context
static void run_job(neo_gpu_batch* b, Worker& w, Job* j) {
    int rc = NEO_OK;
    std::string err;  // a copy: finishing the request may overwrite the context's message
    try {
        rc = j->mem ? neo_gpu_shard_create_mem(w.ctx, &j->ccs->d, j->m_in, j->k_rho, j->label.c_str(), &j->mem->d,
                                               &j->shard)
                    : neo_gpu_shard_create(w.ctx, &j->ccs->d, j->m_in, j->k_rho, j->label.c_str(), &j->shard);
        const uint64_t m = j->ccs->d.m;
        while (rc == NEO_OK && j->steps_done < j->n_steps) {
            if (j->cancel.load(std::memory_order_relaxed)) {
                rc = NEO_ERR_CANCELLED;
                break;
            }
            if (j->steps_done > 0 && j->steps_done < j->inits.size()) {
                auto& st = j->inits[j->steps_done];
                for (uint32_t i = 0; rc == NEO_OK && i < st.size(); i++)
                    rc = neo_gpu_shard_set_twist_init(j->shard, i, st[i].first.size(), st[i].first.data(),
                                                      st[i].second.data());
            }
            if (rc != NEO_OK) break;
            uint64_t len = 0;
            const uint64_t* zs = j->z.size() > m ? j->z.data() + (uint64_t)j->steps_done * m : j->z.data();
            rc = neo_gpu_shard_fold_step(j->shard, zs, nullptr, 0, &len);
            if (rc == NEO_OK) j->steps_done++;
        }
        if (rc == NEO_ERR_CANCELLED) err = "cancelled";
        else if (rc != NEO_OK) err = neo_gpu_last_error(w.ctx);
    } catch (const std::bad_alloc&) {  // the request fails, the worker and the engine go on
        rc = NEO_ERR_OOM;
        err = "host allocation failed";
    } catch (...) {
        rc = NEO_ERR_INVARIANT;
        err = "exception in the batch worker";
    }
    finish_job(b, j, rc == NEO_OK ? 1 : -rc, rc != NEO_OK ? err.c_str() : nullptr);
}

static void worker_main(neo_gpu_batch* b, size_t wi) {
    Worker& w = b->workers[wi];
    cudaSetDevice(b->device);
    g_alloc_stream = w.ctx->stream;  // this thread's shards allocate and free on its stream, from the pool
    for (;;) {
        Job* j = nullptr;
        {
            std::unique_lock<std::mutex> lk(b->mu);
            b->cv_work.wait(lk, [&] { return b->stop || head_fits_locked(b); });
            if (b->stop) return;
            j = b->pending.front();
            b->pending.pop_front();
            b->reserved += j->footprint;
            j->t_admit = bclock::now();
        }
        run_job(b, w, j);
    }
}

static int neo_gpu_batch_create_impl_abi(int device, uint32_t n_workers, neo_gpu_batch** out) {
    if (!out || n_workers == 0 || n_workers > 256) return NEO_ERR_ARG;
    *out = nullptr;
    auto* b = new neo_gpu_batch();
    b->device = device;
    b->workers.resize(n_workers);
    for (auto& w : b->workers) {
        int rc = neo_gpu_ctx_create(device, &w.ctx);
        if (rc != NEO_OK) {
            for (auto& w2 : b->workers)
                if (w2.ctx) neo_gpu_ctx_destroy(w2.ctx);
            delete b;
            return rc;
        }
    }
    // freed shard buffers stay in the device's memory pool for the next request
    // (returned to the driver only when the engine is idle, see head_fits_locked)
    cudaMemPool_t pool;
    cudaSetDevice(device);
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    for (size_t i = 0; i < b->workers.size(); i++) b->threads.emplace_back(worker_main, b, i);
    *out = b;
    return NEO_OK;
}
extern "C" int neo_gpu_batch_create(int device, uint32_t n_workers, neo_gpu_batch** out) { NEO_ABI_GUARD(neo_gpu_batch_create_impl_abi(device, n_workers, out)) }

static int neo_gpu_batch_set_reserve_impl_abi(neo_gpu_batch* b, uint64_t bytes) {
    if (!b) return NEO_ERR_ARG;
    std::lock_guard<std::mutex> lk(b->mu);
    b->reserve_margin = bytes;
    return NEO_OK;
}
extern "C" int neo_gpu_batch_set_reserve(neo_gpu_batch* b, uint64_t bytes) { NEO_ABI_GUARD(neo_gpu_batch_set_reserve_impl_abi(b, bytes)) }

static int submit_impl(neo_gpu_batch* b, const neo_ccs_desc* ccs, const neo_mem_desc* mem, const uint64_t* z,
                       uint32_t n_steps, uint32_t m_in, uint32_t k_rho, const char* app_label, uint64_t* job_id,
                       bool per_step = false, const neo_mem_init* inits = nullptr) {
    if (!b || !ccs || !z || !app_label || !job_id || n_steps == 0 || ccs->m == 0) return NEO_ERR_ARG;
    auto j = std::make_unique<Job>();
    j->ccs = std::make_unique<CcsCopy>(ccs);
    if (mem && (mem->n_shout || mem->n_twist)) j->mem = std::make_unique<MemCopy>(mem);
    j->z.assign(z, z + (per_step ? (uint64_t)n_steps : 1ull) * ccs->m);
    const uint32_t n_twist = j->mem ? j->mem->d.n_twist : 0;
    if (inits && n_twist) {
        j->inits.resize(n_steps);
        for (uint32_t st = 1; st < n_steps; st++)
            for (uint32_t i = 0; i < n_twist; i++) {
                const neo_mem_init& e = inits[(uint64_t)st * n_twist + i];
                if (e.n_init && (!e.addr || !e.val)) return NEO_ERR_ARG;
                j->inits[st].emplace_back(std::vector<uint64_t>(e.addr, e.addr + e.n_init),
                                          std::vector<uint64_t>(e.val, e.val + e.n_init));
            }
    }
    j->n_steps = n_steps;
    j->m_in = m_in;
    j->k_rho = k_rho;
    j->label = app_label;
    j->footprint = shard_footprint(ccs->m, k_rho);
    if (j->mem) {
        // decoded bus columns (this and the previous step), oracle tables, val-lane planes
        uint64_t cols = 0;
        for (auto& s : j->mem->shout) cols += s.ell_addr + 2;
        for (auto& t : j->mem->twist) cols += 2 * t.ell_addr + 5;
        j->footprint += 8 * cols * ccs->n * 16 + (uint64_t)(k_rho + 2) * 54 * ccs->m + (64ull << 20);
    }
    j->t_submit = bclock::now();
    std::lock_guard<std::mutex> lk(b->mu);
    j->id = b->jobs.size();
    *job_id = j->id;
    b->pending.push_back(j.get());
    b->jobs.push_back(std::move(j));
    b->unfinished++;
    b->cv_work.notify_all();
    return NEO_OK;
}

static int neo_gpu_batch_submit_impl_abi(neo_gpu_batch* b, const neo_ccs_desc* ccs, const uint64_t* z, uint32_t n_steps,
                                    uint32_t m_in, uint32_t k_rho, const char* app_label, uint64_t* job_id) {
    return submit_impl(b, ccs, nullptr, z, n_steps, m_in, k_rho, app_label, job_id);
}
extern "C" int neo_gpu_batch_submit(neo_gpu_batch* b, const neo_ccs_desc* ccs, const uint64_t* z, uint32_t n_steps,
                                    uint32_t m_in, uint32_t k_rho, const char* app_label, uint64_t* job_id) { NEO_ABI_GUARD(neo_gpu_batch_submit_impl_abi(b, ccs, z, n_steps, m_in, k_rho, app_label, job_id)) }

static int neo_gpu_batch_submit_mem_impl_abi(neo_gpu_batch* b, const neo_ccs_desc* ccs, const neo_mem_desc* mem,
                                        const uint64_t* z, uint32_t n_steps, uint32_t m_in, uint32_t k_rho,
                                        const char* app_label, uint64_t* job_id) {
    return submit_impl(b, ccs, mem, z, n_steps, m_in, k_rho, app_label, job_id);
}
extern "C" int neo_gpu_batch_submit_mem(neo_gpu_batch* b, const neo_ccs_desc* ccs, const neo_mem_desc* mem,
                                        const uint64_t* z, uint32_t n_steps, uint32_t m_in, uint32_t k_rho,
                                        const char* app_label, uint64_t* job_id) { NEO_ABI_GUARD(neo_gpu_batch_submit_mem_impl_abi(b, ccs, mem, z, n_steps, m_in, k_rho, app_label, job_id)) }

static int neo_gpu_batch_submit_chunks_impl_abi(neo_gpu_batch* b, const neo_ccs_desc* ccs, const neo_mem_desc* mem,
                                           const uint64_t* zs, const neo_mem_init* inits, uint32_t n_steps,
                                           uint32_t m_in, uint32_t k_rho, const char* app_label, uint64_t* job_id) {
    return submit_impl(b, ccs, mem, zs, n_steps, m_in, k_rho, app_label, job_id, true, inits);
}
extern "C" int neo_gpu_batch_submit_chunks(neo_gpu_batch* b, const neo_ccs_desc* ccs, const neo_mem_desc* mem,
                                           const uint64_t* zs, const neo_mem_init* inits, uint32_t n_steps,
                                           uint32_t m_in, uint32_t k_rho, const char* app_label, uint64_t* job_id) { NEO_ABI_GUARD(neo_gpu_batch_submit_chunks_impl_abi(b, ccs, mem, zs, inits, n_steps, m_in, k_rho, app_label, job_id)) }

static int neo_gpu_batch_wait_all_impl_abi(neo_gpu_batch* b, double timeout_ms) {
    if (!b) return NEO_ERR_ARG;
    std::unique_lock<std::mutex> lk(b->mu);
    bool ok = b->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms),
                                  [&] { return b->unfinished == 0; });
    return ok ? NEO_OK : NEO_ERR_CUDA;
}
extern "C" int neo_gpu_batch_wait_all(neo_gpu_batch* b, double timeout_ms) { NEO_ABI_GUARD(neo_gpu_batch_wait_all_impl_abi(b, timeout_ms)) }

/* times3: [submit -> done ms, submit -> admit ms, submit time since batch creation ms] */
static int neo_gpu_batch_job_info_impl_abi(neo_gpu_batch* b, uint64_t job_id, double* times3, uint64_t* tr_state8,
                                      int* status) {
    if (!b) return NEO_ERR_ARG;
    std::lock_guard<std::mutex> lk(b->mu);
    if (job_id >= b->jobs.size()) return NEO_ERR_ARG;
    Job* j = b->jobs[job_id].get();
    if (status) *status = j->status;
    if (times3) {
        using ms = std::chrono::duration<double, std::milli>;
        times3[0] = j->status ? ms(j->t_done - j->t_submit).count() : -1.0;
        times3[1] = ms(j->t_admit - j->t_submit).count();
        times3[2] = ms(j->t_submit - b->t0).count();
    }
    if (tr_state8) memcpy(tr_state8, j->tr_state, 64);
    return NEO_OK;
}
extern "C" int neo_gpu_batch_job_info(neo_gpu_batch* b, uint64_t job_id, double* times3, uint64_t* tr_state8,
                                      int* status) { NEO_ABI_GUARD(neo_gpu_batch_job_info_impl_abi(b, job_id, times3, tr_state8, status)) }

static int neo_gpu_batch_job_error_impl_abi(neo_gpu_batch* b, uint64_t job_id, char* buf, uint64_t cap) {
    if (!b || !buf || cap == 0) return NEO_ERR_ARG;
    std::lock_guard<std::mutex> lk(b->mu);
    if (job_id >= b->jobs.size()) return NEO_ERR_ARG;
    const std::string& e = b->jobs[job_id]->error;
    const size_t n = std::min<size_t>(e.size(), cap - 1);
    memcpy(buf, e.data(), n);
    buf[n] = 0;
    return NEO_OK;
}
extern "C" int neo_gpu_batch_job_error(neo_gpu_batch* b, uint64_t job_id, char* buf, uint64_t cap) { NEO_ABI_GUARD(neo_gpu_batch_job_error_impl_abi(b, job_id, buf, cap)) }

static int neo_gpu_batch_cancel_impl_abi(neo_gpu_batch* b, uint64_t job_id) {
    if (!b) return NEO_ERR_ARG;
    std::lock_guard<std::mutex> lk(b->mu);
    if (job_id >= b->jobs.size()) return NEO_ERR_ARG;
    Job* j = b->jobs[job_id].get();
    auto it = std::find(b->pending.begin(), b->pending.end(), j);
    if (it != b->pending.end()) {  // queued: finish it here, it never reaches a worker
        b->pending.erase(it);
        j->status = -NEO_ERR_CANCELLED;
        j->error = "cancelled";
        j->t_admit = j->t_done = bclock::now();
        b->unfinished--;
        b->cv_work.notify_all();  // the new head of the queue may fit now
        b->cv_done.notify_all();
    } else if (j->status == 0) {
        j->cancel.store(true, std::memory_order_relaxed);  // running: stops before its next step
    }
    return NEO_OK;
}
extern "C" int neo_gpu_batch_cancel(neo_gpu_batch* b, uint64_t job_id) { NEO_ABI_GUARD(neo_gpu_batch_cancel_impl_abi(b, job_id)) }

static int neo_gpu_batch_destroy_impl_abi(neo_gpu_batch* b) {
    if (!b) return NEO_ERR_ARG;
    {
        std::lock_guard<std::mutex> lk(b->mu);
        b->stop = true;
        b->cv_work.notify_all();
    }
    for (auto& t : b->threads) t.join();  // running requests finish; queued ones never start
    for (auto& w : b->workers) neo_gpu_ctx_destroy(w.ctx);
    delete b;
    return NEO_OK;
}
extern "C" int neo_gpu_batch_destroy(neo_gpu_batch* b) { NEO_ABI_GUARD(neo_gpu_batch_destroy_impl_abi(b)) }

extern "C" uint64_t neo_gpu_batch_kernel_launches(const neo_gpu_batch* b) {
    if (!b) return 0;
    uint64_t n = 0;
    for (auto& w : b->workers) n += neo_gpu_kernel_launches(w.ctx);
    return n;
}
