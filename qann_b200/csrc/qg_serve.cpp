// The serving loop: continuous batching of single-query requests over one
// device-resident index. No counterpart in the reference, which answers each
// query_batch call on the calling threads (reference bindings/python_bindings.cpp:600-648).
//
// Requests (a query with its own k, nprobe and optional filter) enter a FIFO
// queue. `slots` worker threads, each with its own CUDA stream, take the
// oldest waiting requests as soon as they are free, up to max_batch at a
// time and only while the device memory of every batch in flight (estimated
// per request: its query, coarse scores, probe lists, tables, candidate
// buffers and filter) stays within the budget. A batch runs as one mixed
// search (search_mixed: one coarse step, one scan and one re-rank for all of
// it), so requests that arrive while others are on the GPU start as soon as a
// slot frees, and batches on different slots overlap on the device. Each
// request's results are the ones it gets searched alone. Over a RefineIndex,
// requests whose filter is narrow enough for its exact direct scan (at most
// 6 * nlist allowed slots) queue in a lane of their own with one more worker,
// so that approximate batches never wait for those scans.
#include "../../include/qann_gpu.h"

#include "qg_index.h"
#include "qg_ops.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <limits>
#include <mutex>
#include <thread>
#include <unordered_map>

namespace qg {

namespace {

double now_us() {
    using namespace std::chrono;
    return duration<double, std::micro>(steady_clock::now().time_since_epoch()).count();
}

struct ServeRequest {
    std::vector<float> q;
    MixedQuery mq;
    std::shared_ptr<const SlotBits> filter;   // keeps mq.filter alive
    double t_arrive = 0, t_done = 0;
    size_t bytes = 0;
    int status = -1;   // -1 while pending, then a QG_* status
    bool claimed = false;   // a thread is waiting on it
    std::string err;
    std::vector<int64_t> ids;
    std::vector<float> d;
};

} // namespace

class Server {
public:
    Server(std::shared_ptr<IndexObj> idx, int slots, int max_batch, size_t budget)
        : idx_(std::move(idx)), max_batch_(max_batch), budget_(budget) {
        IndexObj* ivf = idx_.get();
        if (idx_->kind == Kind::Refine) ivf = static_cast<RefineObj&>(*idx_).base.get();
        if (ivf->kind == Kind::IVF) {
            const IVFModel& M = static_cast<IVFObj&>(*ivf).model;
            nlist_ = M.nlist;
            nprobe_ = M.nprobe;
            m_ = M.pq.m;
        }
        if (idx_->kind == Kind::Refine) k_factor_ = static_cast<RefineObj&>(*idx_).k_factor;
        direct_lane_ = idx_->kind == Kind::Refine && nlist_ > 0;
        for (int s = 0; s < slots; ++s) workers_.emplace_back([this] { worker(0); });
        if (direct_lane_) workers_.emplace_back([this] { worker(1); });
    }

    ~Server() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        for (auto& cv : cv_in_) cv.notify_all();
        for (auto& t : workers_) t.join();
        std::unique_lock<std::mutex> lk(mu_);
        for (auto& [id, r] : reqs_)
            if (r->status < 0) {
                r->status = QG_RUNTIME_ERROR;
                r->err = "server stopped";
            }
        cv_out_.notify_all();
        // threads still inside wait() hold references to mu_ and cv_out_:
        // let every one of them take its request and leave before the
        // members are destroyed
        cv_out_.wait(lk, [&] { return waiters_ == 0; });
    }

    size_t dim() const { return idx_->dim(); }
    size_t nlist() const { return nlist_; }
    IndexObj& index() { return *idx_; }

    // A registered filter is uploaded once, here, and its device copy serves
    // every batch that uses it (without a usable device, batches upload the
    // bitmap themselves, as for unregistered filters). A filter narrow enough
    // for a RefineIndex's direct scan (at most 6 * nlist allowed slots) also
    // keeps its allowed slots, ascending, on the device, so that the scan
    // need not list them from the bitmap on every batch.
    int add_filter(std::shared_ptr<const SlotBits> f) {
        auto reg = std::make_shared<Registered>();
        try {
            cudaStream_t st = resident_stream();
            reg->dev.alloc(std::max<size_t>(1, f->words.size()), st);
            QG_CUDA(cudaMemcpyAsync(reg->dev.get(), f->words.data(), f->words.size() * sizeof(uint64_t),
                                    cudaMemcpyHostToDevice, st));
            std::vector<uint32_t> slots;
            if (idx_->kind == Kind::Refine && nlist_ > 0 && f->count > 0 && f->count <= 6 * nlist_) {
                slots.reserve(f->count);
                for (size_t w = 0; w < f->words.size(); ++w)
                    for (uint64_t bits = f->words[w]; bits; bits &= bits - 1)
                        slots.push_back(static_cast<uint32_t>(w * 64 + __builtin_ctzll(bits)));
                if (slots.size() == f->count) {
                    reg->slots.alloc(slots.size(), st);
                    QG_CUDA(cudaMemcpyAsync(reg->slots.get(), slots.data(), slots.size() * 4, cudaMemcpyHostToDevice,
                                            st));
                }
            }
            QG_CUDA(cudaStreamSynchronize(st));
        } catch (const Error&) {
            reg->dev = DevBuf<uint64_t>{};
            reg->slots = DevBuf<uint32_t>{};
            (void)cudaGetLastError();
        }
        reg->bits = std::move(f);
        std::lock_guard<std::mutex> g(mu_);
        filters_.push_back(std::move(reg));
        return static_cast<int>(filters_.size() - 1);
    }
    std::shared_ptr<const SlotBits> filter(int id) { return registered(id)->bits; }
    const uint64_t* filter_dev(int id) { return registered(id)->dev.get(); }
    const uint32_t* filter_slots(int id) { return registered(id)->slots.get(); }

    uint64_t submit(const float* q, int k, int nprobe, std::shared_ptr<const SlotBits> f, double t_arrive,
                    const uint64_t* f_dev = nullptr, const uint32_t* f_slots = nullptr) {
        require(k >= 1, "k must be at least 1");
        require(nprobe <= 0 || nlist_ == 0 || static_cast<size_t>(nprobe) <= nlist_, "nprobe must be <= nlist");
        const size_t d = dim();
        if (idx_->metric() == Metric::Cosine)
            require(std::any_of(q, q + d, [](float v) { return v != 0.0f; }), "cosine metric needs non-zero vectors");
        auto r = std::make_unique<ServeRequest>();
        r->q.assign(q, q + d);
        r->mq.k = k;
        r->mq.nprobe = nprobe;
        r->filter = std::move(f);
        r->mq.filter = r->filter.get();
        r->mq.filter_dev = r->filter ? f_dev : nullptr;
        r->mq.filter_slots_dev = r->filter ? f_slots : nullptr;
        r->t_arrive = t_arrive;
        r->bytes = footprint(*r);
        const size_t r_filter_count = r->filter ? r->filter->count : SIZE_MAX;
        std::lock_guard<std::mutex> g(mu_);
        const uint64_t id = next_++;
        reqs_.emplace(id, std::move(r));
        // narrow filters of a RefineIndex over IVF take the exact direct scan
        // (RefineIndex::use_direct): their own lane and worker, so that a
        // batch of approximate searches never waits for one
        const int lane = direct_lane_ && r_filter_count <= 6 * nlist_ && r_filter_count > 0 ? 1 : 0;
        queue_[lane].push_back(id);
        cv_in_[lane].notify_one();
        return id;
    }

    // Waits for a request and takes its results (k entries each).
    // One thread waits per ticket. The request is owned by the map until
    // then; no iterator is held across the wait, because submit() may
    // rehash the map while this thread sleeps.
    void wait(uint64_t id, int64_t* ids, float* d, double* latency_us) {
        std::unique_lock<std::mutex> lk(mu_);
        auto it = reqs_.find(id);
        require(it != reqs_.end(), "unknown ticket");
        ServeRequest* r = it->second.get();
        require(!r->claimed, "another thread is already waiting on this ticket");
        r->claimed = true;
        ++waiters_;
        cv_out_.wait(lk, [&] { return r->status >= 0; });
        auto jt = reqs_.find(id);
        std::unique_ptr<ServeRequest> own = std::move(jt->second);
        reqs_.erase(jt);
        if (--waiters_ == 0 && stop_) cv_out_.notify_all();
        lk.unlock();
        if (own->status != QG_OK) throw Error(own->status, own->err);
        if (ids) std::copy(own->ids.begin(), own->ids.end(), ids);
        if (d) std::copy(own->d.begin(), own->d.end(), d);
        if (latency_us) *latency_us = own->t_done - own->t_arrive;
    }

    void stats(int64_t* completed, int64_t* batches, int64_t* peak_bytes) {
        std::lock_guard<std::mutex> g(mu_);
        if (completed) *completed = completed_;
        if (batches) *batches = batches_;
        if (peak_bytes) *peak_bytes = static_cast<int64_t>(peak_);
    }

private:
    struct Registered {
        std::shared_ptr<const SlotBits> bits;
        DevBuf<uint64_t> dev;
        DevBuf<uint32_t> slots;   // narrow filters of a RefineIndex: the allowed slots, ascending
    };
    std::shared_ptr<Registered> registered(int id) {
        std::lock_guard<std::mutex> g(mu_);
        require(id >= 0 && static_cast<size_t>(id) < filters_.size(), "unknown filter id");
        return filters_[id];
    }

    // Device bytes one request adds to a batch: query copies, the coarse
    // scores (every list ranked when filtered), probe lists and terms, the
    // query's tables, candidate lists per probe chunk and after the merge,
    // results, and its filter's bitmap.
    size_t footprint(const ServeRequest& r) const {
        const size_t d = dim();
        const size_t np = r.mq.nprobe > 0 ? static_cast<size_t>(r.mq.nprobe) : std::max<size_t>(nprobe_, 1);
        const size_t kp = static_cast<size_t>(r.mq.k) * k_factor_;
        size_t b = 3 * d * 4 + nlist_ * 4 + np * 12 + m_ * 16 * 4 + 256;
        b += kp * 12 * (2 + (np + 15) / 16) + static_cast<size_t>(r.mq.k) * 12;
        if (r.filter) b += nlist_ * 12 + (r.mq.filter_dev ? 0 : r.filter->words.size() * 8);
        return b;
    }

    // lane 0: every request but the narrow-filter ones; lane 1: those (see submit)
    void worker(int lane) {
        cudaStream_t st = nullptr, st2 = nullptr;   // st2: a mixed batch's larger k' class, at the same time
        if (cudaSetDevice(idx_->device) != cudaSuccess ||
            cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
            st = nullptr;
        if (st && cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking) != cudaSuccess) st2 = nullptr;
        keep_pool_memory();
        const size_t d = dim();
        std::vector<ServeRequest*> b;
        std::vector<float> q;
        std::vector<MixedQuery> mq;
        std::vector<int64_t> ids;
        std::vector<float> dist;
        for (;;) {
            b.clear();
            size_t bytes = 0;
            {
                std::unique_lock<std::mutex> lk(mu_);
                std::deque<uint64_t>& queue = queue_[lane];
                cv_in_[lane].wait(lk, [&] {
                    return stop_ || (!queue.empty() &&
                                     (in_flight_ == 0 || in_flight_ + reqs_.at(queue.front())->bytes <= budget_));
                });
                if (stop_) break;
                while (!queue.empty() && b.size() < static_cast<size_t>(max_batch_)) {
                    ServeRequest* r = reqs_.at(queue.front()).get();
                    if ((in_flight_ > 0 || !b.empty()) && in_flight_ + bytes + r->bytes > budget_) break;
                    b.push_back(r);
                    bytes += r->bytes;
                    queue.pop_front();
                }
                in_flight_ += bytes;
                peak_ = std::max(peak_, in_flight_);
            }
            const size_t nb = b.size();
            size_t kmax = 0;
            q.resize(nb * d);
            mq.resize(nb);
            for (size_t j = 0; j < nb; ++j) {
                std::copy(b[j]->q.begin(), b[j]->q.end(), q.begin() + j * d);
                mq[j] = b[j]->mq;
                kmax = std::max(kmax, static_cast<size_t>(b[j]->mq.k));
            }
            ids.resize(nb * kmax);
            dist.resize(nb * kmax);
            int status = QG_OK;
            std::string err;
            try {
                require(st != nullptr, "could not create a CUDA stream for the server", kCudaError);
                std::shared_lock<std::shared_mutex> lk(idx_->mu);
                std::shared_lock<std::shared_mutex> lb;
                if (idx_->kind == Kind::Refine) lb = std::shared_lock<std::shared_mutex>(static_cast<RefineObj&>(*idx_).base->mu);
                search_mixed(*idx_, q.data(), nb, mq.data(), kmax, ids.data(), dist.data(), st, st2);
            } catch (const Error& e) {
                status = e.status;
                err = e.what();
            } catch (const std::exception& e) {
                status = QG_RUNTIME_ERROR;
                err = e.what();
            }
            const double t = now_us();
            {
                std::lock_guard<std::mutex> g(mu_);
                for (size_t j = 0; j < nb; ++j) {
                    ServeRequest* r = b[j];
                    const size_t k = static_cast<size_t>(r->mq.k);
                    r->ids.assign(ids.begin() + j * kmax, ids.begin() + j * kmax + k);
                    r->d.assign(dist.begin() + j * kmax, dist.begin() + j * kmax + k);
                    r->t_done = t;
                    r->err = err;
                    r->status = status;
                }
                in_flight_ -= bytes;
                completed_ += static_cast<int64_t>(nb);
                ++batches_;
            }
            cv_out_.notify_all();
            for (auto& cv : cv_in_) cv.notify_all();
        }
        if (st2) cudaStreamDestroy(st2);
        if (st) cudaStreamDestroy(st);
    }

    std::shared_ptr<IndexObj> idx_;
    int max_batch_;
    size_t budget_;
    size_t nlist_ = 0, nprobe_ = 0, m_ = 0, k_factor_ = 1;
    std::mutex mu_;
    std::condition_variable cv_in_[2], cv_out_;
    std::deque<uint64_t> queue_[2];   // the lanes (see worker)
    bool direct_lane_ = false;
    std::unordered_map<uint64_t, std::unique_ptr<ServeRequest>> reqs_;
    std::vector<std::shared_ptr<Registered>> filters_;
    uint64_t next_ = 1;
    size_t in_flight_ = 0, peak_ = 0;
    int waiters_ = 0;   // threads inside wait()
    int64_t completed_ = 0, batches_ = 0;
    bool stop_ = false;
    std::vector<std::thread> workers_;
};

} // namespace qg

using namespace qg;

struct qg_server {
    std::unique_ptr<Server> s;
};

namespace {

template <class F>
int served(F&& f) {
    try {
        f();
        return QG_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.status;
    } catch (const std::bad_alloc&) {
        set_last_error("out of host memory");
        return QG_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return QG_RUNTIME_ERROR;
    }
}

Server& srv(qg_server* s) {
    require(s && s->s, "null server handle");
    return *s->s;
}

} // namespace

extern "C" {

int qg_server_create(qg_index* h, int slots, int max_batch, size_t mem_budget_bytes, qg_server** out) {
    return served([&] {
        require(h && h->obj && out, "null argument");
        require(slots >= 1 && slots <= 64, "slots must be in 1..64");
        require(max_batch >= 1, "max_batch must be at least 1");
        auto* s = new qg_server;
        s->s = std::make_unique<Server>(h->obj, slots, max_batch, mem_budget_bytes ? mem_budget_bytes : size_t{2} << 30);
        *out = s;
    });
}

int qg_server_add_filter(qg_server* s, const uint64_t* words, size_t nwords, int* filter_id) {
    return served([&] {
        Server& v = srv(s);
        require(words && filter_id, "null argument");
        std::shared_lock<std::shared_mutex> lk(v.index().mu);
        require(nwords * 64 >= v.index().idmap().slots(), "the bitmap must cover every slot of the index");
        auto f = std::make_shared<SlotBits>(v.index().idmap().live(std::vector<uint64_t>(words, words + nwords)));
        lk.unlock();
        *filter_id = v.add_filter(std::move(f));
    });
}

int qg_server_submit(qg_server* s, const float* q, size_t k, int nprobe, const int64_t* allowed, size_t n_allowed,
                     int filter_id, uint64_t* ticket) {
    return served([&] {
        Server& v = srv(s);
        require(q && ticket, "null argument");
        std::shared_ptr<const SlotBits> f;
        if (allowed) {
            std::shared_lock<std::shared_mutex> lk(v.index().mu);
            f = std::make_shared<SlotBits>(v.index().idmap().filter({allowed, n_allowed}));
        }
        const uint64_t* f_dev = nullptr;
        const uint32_t* f_slots = nullptr;
        if (!allowed && filter_id >= 0) {
            f = v.filter(filter_id);
            f_dev = v.filter_dev(filter_id);
            f_slots = v.filter_slots(filter_id);
        }
        *ticket = v.submit(q, static_cast<int>(k), nprobe, std::move(f), now_us(), f_dev, f_slots);
    });
}

int qg_server_wait(qg_server* s, uint64_t ticket, int64_t* out_ids, float* out_dists, double* latency_us) {
    return served([&] { srv(s).wait(ticket, out_ids, out_dists, latency_us); });
}

int qg_server_replay(qg_server* s, const float* q, size_t nq, const int32_t* k, const int32_t* nprobe,
                     const int32_t* filter_id, const double* arrival_us, size_t kmax, int64_t* out_ids,
                     float* out_dists, double* latency_us) {
    return served([&] {
        Server& v = srv(s);
        require(q && k && arrival_us && out_ids && out_dists && latency_us, "null argument");
        const size_t d = v.dim();
        for (size_t i = 0; i < nq; ++i) require(k[i] >= 1 && static_cast<size_t>(k[i]) <= kmax, "k out of range");
        std::vector<std::shared_ptr<const SlotBits>> fs(nq);
        std::vector<const uint64_t*> fdev(nq, nullptr);
        std::vector<const uint32_t*> fslots(nq, nullptr);
        for (size_t i = 0; i < nq; ++i)
            if (filter_id && filter_id[i] >= 0) {
                fs[i] = v.filter(filter_id[i]);
                fdev[i] = v.filter_dev(filter_id[i]);
                fslots[i] = v.filter_slots(filter_id[i]);
            }
        std::vector<uint64_t> tickets(nq);
        // open loop: request i enters at t0 + arrival_us[i] whatever the state
        // of the others; its latency runs from that moment to its results
        const double t0 = now_us() + 1000.0;
        for (size_t i = 0; i < nq; ++i) {
            const double due = t0 + arrival_us[i];
            for (double t = now_us(); t < due; t = now_us()) {
                if (due - t > 300.0) std::this_thread::sleep_for(std::chrono::microseconds(static_cast<int64_t>(due - t - 200.0)));
            }
            tickets[i] = v.submit(q + i * d, k[i], nprobe ? nprobe[i] : 0, fs[i], due, fdev[i], fslots[i]);
        }
        std::vector<int64_t> ids(kmax);
        std::vector<float> dd(kmax);
        for (size_t i = 0; i < nq; ++i) {
            std::fill(out_ids + i * kmax, out_ids + (i + 1) * kmax, int64_t{-1});
            std::fill(out_dists + i * kmax, out_dists + (i + 1) * kmax, std::numeric_limits<float>::infinity());
            v.wait(tickets[i], out_ids + i * kmax, out_dists + i * kmax, latency_us + i);
        }
    });
}

int qg_server_stats(qg_server* s, int64_t* completed, int64_t* batches, int64_t* peak_bytes) {
    return served([&] { srv(s).stats(completed, batches, peak_bytes); });
}

void qg_server_free(qg_server* s) { delete s; }

} // extern "C"
