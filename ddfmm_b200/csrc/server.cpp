// Matvec server (see server.hpp).
#include "server.hpp"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <stdexcept>

namespace ddfmm {

#define SCK(x)                                                                                     \
    do {                                                                                           \
        cudaError_t e_ = (x);                                                                      \
        if (e_ != cudaSuccess)                                                                     \
            throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " (" + \
                                     #x + ")");                                                    \
    } while (0)

namespace {
// Host copies of a tick (densities into pinned staging, values out of it): split
// into pieces of at most 1 MiB and spread over up to 8 threads; one thread when
// the tick moves less than 1 MiB.
struct Copy {
    void* dst;
    const void* src;
    size_t bytes;
};
void parallel_copy(const std::vector<Copy>& jobs) {
    constexpr size_t kPiece = 1 << 20;
    std::vector<Copy> pieces;
    size_t total = 0;
    for (const Copy& c : jobs) {
        total += c.bytes;
        for (size_t o = 0; o < c.bytes; o += kPiece)
            pieces.push_back(Copy{static_cast<char*>(c.dst) + o, static_cast<const char*>(c.src) + o,
                                  std::min(kPiece, c.bytes - o)});
    }
    const size_t nt = std::min<size_t>({8, std::max(1u, std::thread::hardware_concurrency()), pieces.size()});
    if (total < kPiece || nt <= 1) {
        for (const Copy& c : pieces) std::memcpy(c.dst, c.src, c.bytes);
        return;
    }
    std::vector<std::thread> th;
    for (size_t t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            for (size_t i = t; i < pieces.size(); i += nt) std::memcpy(pieces[i].dst, pieces[i].src, pieces[i].bytes);
        });
    for (auto& x : th) x.join();
}
}  // namespace

double Server::now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

Server::Server(int device, size_t budget_bytes) : device_(device), budget_(budget_bytes) {
    SCK(cudaSetDevice(device_));
    SCK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    admit_thread_ = std::thread([this] { admission_loop(); });
    serve_thread_ = std::thread([this] { serving_loop(); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_work_.notify_all();
    cv_admit_.notify_all();
    if (admit_thread_.joinable()) admit_thread_.join();
    if (serve_thread_.joinable()) serve_thread_.join();
    cudaSetDevice(device_);
    if (stream_) cudaStreamSynchronize(stream_);
    batch_.reset();
    for (auto& kv : entries_) {
        Entry& e = *kv.second;
        if (e.h_den) cudaFreeHost(e.h_den);
        if (e.h_val) cudaFreeHost(e.h_val);
        e.s.reset();
    }
    if (d_active_) cudaFree(d_active_);
    if (h_active_) cudaFreeHost(h_active_);
    if (stream_) cudaStreamDestroy(stream_);
}

int Server::add_session(SessionSpec spec) {
    if (spec.n <= 0 || spec.pos.size() != 3 * (size_t)spec.n) throw std::invalid_argument("need n > 0 points");
    spec.params.precision = PRECISION_MIXED;
    spec.params.device = device_;
    std::lock_guard<std::mutex> lk(mu_);
    const int sid = next_sid_++;
    std::unique_ptr<Entry> e(new Entry());
    e->spec = std::move(spec);
    entries_[sid] = std::move(e);
    waiting_.push_back(sid);
    cv_admit_.notify_all();
    return sid;
}

int Server::state(int sid, std::string* why) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = entries_.find(sid);
    if (it == entries_.end()) return -1;
    if (why) *why = it->second->why;
    return it->second->state;
}

void Server::remove_session(int sid) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = entries_.find(sid);
    if (it == entries_.end()) throw std::invalid_argument("unknown session");
    Entry& e = *it->second;
    if (e.state == WAITING) {
        waiting_.erase(std::remove(waiting_.begin(), waiting_.end(), sid), waiting_.end());
        e.state = REMOVED;
        return;
    }
    if (e.state == ADMITTED) {
        e.removing = true;  // the serving thread drops it between ticks
        cv_work_.notify_all();
    }
}

long long Server::submit(int sid, const std::complex<float>* den, std::complex<float>* val) {
    if (!den || !val) throw std::invalid_argument("den / val is NULL");
    std::lock_guard<std::mutex> lk(mu_);
    auto it = entries_.find(sid);
    if (it == entries_.end()) throw std::invalid_argument("unknown session");
    Entry& e = *it->second;
    if (e.state == REJECTED || e.state == REMOVED || e.state == FAILED || e.removing)
        throw std::invalid_argument("session is not being served: " + e.why);
    const long long t = next_ticket_++;
    e.queue.push_back(Request{t, den, val, now()});
    cv_work_.notify_all();
    return t;
}

int Server::poll(long long ticket) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = done_.find(ticket);
    if (it == done_.end()) return 1;
    return it->second;
}

int Server::wait(long long ticket, double timeout_s) {
    std::unique_lock<std::mutex> lk(mu_);
    const auto until = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
    while (!done_.count(ticket)) {
        if (cv_done_.wait_until(lk, until) == std::cv_status::timeout && !done_.count(ticket)) return 1;
    }
    const int r = done_[ticket];
    done_.erase(ticket);
    if (r != 0) {
        std::string why = failures_[ticket];
        failures_.erase(ticket);
        throw std::runtime_error(why);
    }
    return 0;
}

ServerStats Server::stats(bool reset) {
    std::lock_guard<std::mutex> lk(mu_);
    ServerStats s;
    s.requests = (long long)lat_ms_.size();
    s.ticks = ticks_;
    s.mean_batch = ticks_ ? (double)reqs_in_ticks_ / ticks_ : 0.0;
    s.busy_s = busy_s_;
    if (!lat_ms_.empty()) {
        std::vector<double> v(lat_ms_);
        std::sort(v.begin(), v.end());
        auto pct = [&](double q) { return v[std::min(v.size() - 1, (size_t)(q * (v.size() - 1) + 0.5))]; };
        s.p50_ms = pct(0.50);
        s.p99_ms = pct(0.99);
        s.max_ms = v.back();
    }
    s.used_bytes = used_ + DevChunk::live_bytes(device_);
    for (auto& kv : entries_) {
        if (kv.second->state == ADMITTED) s.admitted++;
        if (kv.second->state == WAITING) s.waiting++;
    }
    if (reset) {
        lat_ms_.clear();
        ticks_ = reqs_in_ticks_ = 0;
        busy_s_ = 0;
    }
    return s;
}

// ---------------------------------------------------------------- admission
void Server::admission_loop() {
    cudaSetDevice(device_);
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
        cv_admit_.wait(lk, [&] { return stop_ || (!waiting_.empty() && !blocked_); });
        if (stop_) return;
        const int sid = waiting_.front();
        Entry* e = entries_[sid].get();
        lk.unlock();
        std::unique_ptr<Session> s;
        std::string err;
        try {
            const SessionSpec& sp = e->spec;
            s.reset(new Session(sp.pos.data(), sp.n, sp.params, sp.ld, sp.hd));
        } catch (const std::exception& ex) {
            err = ex.what();
        }
        float2 *hd = nullptr, *hv = nullptr;
        if (s && (cudaMallocHost(&hd, sizeof(float2) * e->spec.n) != cudaSuccess ||
                  cudaMallocHost(&hv, sizeof(float2) * e->spec.n) != cudaSuccess)) {
            err = "pinned host staging allocation failed";
            s.reset();
        }
        // device memory: the session's own buffers plus the packed-operator chunks alive
        // on the device, which sessions share and which are counted once
        const size_t total = s ? s->stats().device_bytes : 0;
        const size_t bytes = s ? total - s->chunk_bytes() : 0;
        lk.lock();
        if (waiting_.empty() || waiting_.front() != sid || e->state != WAITING) {  // removed meanwhile
            lk.unlock();
            s.reset();
            if (hd) cudaFreeHost(hd);
            if (hv) cudaFreeHost(hv);
            lk.lock();
            continue;
        }
        if (!s) {
            waiting_.pop_front();
            e->state = FAILED;
            e->why = err;
        } else if (total > budget_) {
            waiting_.pop_front();
            e->state = REJECTED;
            e->why = "needs " + std::to_string(total) + " device bytes, more than the budget of " +
                     std::to_string(budget_);
            lk.unlock();
            s.reset();
            cudaFreeHost(hd);
            cudaFreeHost(hv);
            lk.lock();
        } else if (used_ + bytes + DevChunk::live_bytes(device_) > budget_) {
            // does not fit now: release it and wait for a removal
            blocked_ = true;
            lk.unlock();
            s.reset();
            cudaFreeHost(hd);
            cudaFreeHost(hv);
            lk.lock();
        } else {
            waiting_.pop_front();
            e->s = std::move(s);
            e->bytes = bytes;
            e->h_den = hd;
            e->h_val = hv;
            used_ += bytes;
            e->state = ADMITTED;
            changed_ = true;
            cv_work_.notify_all();
        }
        cv_done_.notify_all();
    }
}

// ---------------------------------------------------------------- serving
void Server::rebuild() {
    batch_.reset();
    slots_.clear();
    std::vector<Session*> ss;
    for (auto& kv : entries_)
        if (kv.second->state == ADMITTED && !kv.second->removing) {
            slots_.push_back(kv.first);
            ss.push_back(kv.second->s.get());
        }
    if (d_active_) cudaFree(d_active_);
    if (h_active_) cudaFreeHost(h_active_);
    d_active_ = nullptr;
    h_active_ = nullptr;
    if (ss.empty()) return;
    batch_.reset(new Batch(ss));
    SCK(cudaMalloc(&d_active_, sizeof(int) * ss.size()));
    SCK(cudaMallocHost(&h_active_, sizeof(int) * ss.size()));
}

void Server::serving_loop() {
    cudaSetDevice(device_);
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
        auto has_work = [&] {
            if (changed_) return true;
            for (auto& kv : entries_)
                if (kv.second->removing || (kv.second->state == ADMITTED && !kv.second->queue.empty())) return true;
            return false;
        };
        cv_work_.wait(lk, [&] { return stop_ || has_work(); });
        if (stop_) {
            for (auto& kv : entries_)
                for (Request& r : kv.second->queue) {
                    done_[r.ticket] = -1;
                    failures_[r.ticket] = "server stopped";
                }
            cv_done_.notify_all();
            return;
        }
        // removals between ticks: fail their queued requests, release their memory
        bool removed = false;
        for (auto& kv : entries_) {
            Entry& e = *kv.second;
            if (!e.removing) continue;
            for (Request& r : e.queue) {
                done_[r.ticket] = -1;
                failures_[r.ticket] = "session removed";
            }
            e.queue.clear();
            batch_.reset();  // it refers to the session's buffers
            e.s.reset();
            if (e.h_den) cudaFreeHost(e.h_den);
            if (e.h_val) cudaFreeHost(e.h_val);
            e.h_den = e.h_val = nullptr;
            used_ -= e.bytes;
            e.bytes = 0;
            e.state = REMOVED;
            e.removing = false;
            removed = true;
        }
        if (removed) {
            changed_ = true;
            blocked_ = false;
            cv_admit_.notify_all();
            cv_done_.notify_all();
        }
        if (changed_) {
            try {
                rebuild();
            } catch (const std::exception& ex) {
                // cannot serve: fail everything queued
                for (auto& kv : entries_)
                    for (Request& r : kv.second->queue) {
                        done_[r.ticket] = -1;
                        failures_[r.ticket] = std::string("batch rebuild failed: ") + ex.what();
                    }
                for (auto& kv : entries_) kv.second->queue.clear();
                cv_done_.notify_all();
            }
            changed_ = false;
        }
        if (!batch_) continue;
        // gather window: sessions of the previous tick usually submit their next
        // request soon after its completion; wait for the stragglers up to 5% of
        // the last tick's duration (0.3 to 5 ms)
        {
            const double win = std::min(5e-3, std::max(3e-4, 0.05 * last_tick_s_));
            const auto until = std::chrono::steady_clock::now() +
                               std::chrono::duration_cast<std::chrono::steady_clock::duration>(
                                   std::chrono::duration<double>(win));
            auto stragglers = [&] {
                for (int sid : prev_tick_) {
                    auto it = entries_.find(sid);
                    if (it != entries_.end() && it->second->state == ADMITTED && !it->second->removing &&
                        it->second->queue.empty())
                        return true;
                }
                return false;
            };
            while (!stop_ && stragglers() && cv_work_.wait_until(lk, until) != std::cv_status::timeout) {
            }
        }
        // the tick: the oldest request of every session that has one
        std::vector<std::pair<int, Request> > tick;  // (slot, request)
        for (size_t i = 0; i < slots_.size(); ++i) {
            Entry& e = *entries_[slots_[i]];
            if (!e.queue.empty()) {
                tick.push_back(std::make_pair((int)i, e.queue.front()));
                e.queue.pop_front();
            }
        }
        if (tick.empty()) continue;
        prev_tick_.clear();
        for (auto& tr : tick) prev_tick_.push_back(slots_[tr.first]);
        std::vector<Entry*> ent(slots_.size(), nullptr);
        for (size_t i = 0; i < slots_.size(); ++i) ent[i] = entries_[slots_[i]].get();
        lk.unlock();
        const double t0 = now();
        std::string err;
        try {
            std::fill(h_active_, h_active_ + slots_.size(), 0);
            std::vector<Copy> in;
            for (auto& tr : tick) {
                Entry& e = *ent[tr.first];
                in.push_back(Copy{e.h_den, tr.second.den, sizeof(float2) * e.spec.n});
            }
            parallel_copy(in);
            for (auto& tr : tick) {
                const int i = tr.first;
                Entry& e = *ent[i];
                SCK(cudaMemcpyAsync(batch_->den(i), e.h_den, sizeof(float2) * e.spec.n, cudaMemcpyHostToDevice,
                                    stream_));
                h_active_[i] = 1;
            }
            SCK(cudaMemcpyAsync(d_active_, h_active_, sizeof(int) * slots_.size(), cudaMemcpyHostToDevice, stream_));
            batch_->run_graph(d_active_, stream_);
            for (auto& tr : tick) {
                Entry& e = *ent[tr.first];
                SCK(cudaMemcpyAsync(e.h_val, batch_->val(tr.first), sizeof(float2) * e.spec.n,
                                    cudaMemcpyDeviceToHost, stream_));
            }
            batch_->check_error(stream_);  // synchronises the stream
            std::vector<Copy> out;
            for (auto& tr : tick) {
                Entry& e = *ent[tr.first];
                out.push_back(Copy{tr.second.val, e.h_val, sizeof(float2) * e.spec.n});
            }
            parallel_copy(out);
        } catch (const std::exception& ex) {
            err = ex.what();
        }
        const double t1 = now();
        lk.lock();
        last_tick_s_ = t1 - t0;
        ticks_++;
        reqs_in_ticks_ += (long long)tick.size();
        busy_s_ += t1 - t0;
        for (auto& tr : tick) {
            if (err.empty()) {
                done_[tr.second.ticket] = 0;
                lat_ms_.push_back((t1 - tr.second.t_submit) * 1e3);
            } else {
                done_[tr.second.ticket] = -1;
                failures_[tr.second.ticket] = err;
            }
        }
        cv_done_.notify_all();
    }
}

}  // namespace ddfmm
