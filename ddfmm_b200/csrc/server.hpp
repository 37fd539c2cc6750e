// Matvec server: sessions (fixed geometry, resident trees, operators and
// buffers) admitted against a device-memory budget, and a request loop that
// batches pending matvecs across sessions.
//
// Continuous batching: the serving thread runs ticks.  A tick takes the
// oldest pending request of every admitted session that has one, copies
// their densities in (host copies into pinned staging split over up to 8
// threads), runs one masked batch matvec (Batch::run_graph: all of
// the tick's sessions in the same merged launches), copies the values out and
// completes the requests.  Requests that arrive during a tick are taken by
// the next one, so work of sessions that become busy at different times
// shares the device as soon as the current tick ends.  Before a tick the
// serving thread waits briefly for sessions of the previous tick that have
// not yet sent their next request (a client answers a completion with a new
// request soon after, but client threads that share an interpreter lock take
// turns): at most 5% of the last tick's duration, between 0.3 and 5 ms.
//
// Admission: add_session queues a session; an admission thread creates it
// (tree, operators, device buffers: seconds for large ones, off the serving
// thread) and admits it if the device bytes of the admitted sessions plus
// its own stay within the budget (packed operators shared through the
// process-wide cache are counted once).  A session that does not fit is released
// and waits, in order, until a removal frees memory; one larger than the
// whole budget is rejected.
#pragma once
#include <complex>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "batch.hpp"
#include "session.hpp"

namespace ddfmm {

struct SessionSpec {
    std::vector<double> pos;  // 3n
    int n = 0;
    SessionParams params;     // precision is forced to the mixed form
    std::string ld, hd;
};

struct ServerStats {
    long long requests = 0;  // completed
    long long ticks = 0;
    double mean_batch = 0;   // requests per tick
    double p50_ms = 0, p99_ms = 0, max_ms = 0;  // submit -> completion
    double busy_s = 0;       // time spent in ticks
    size_t used_bytes = 0;
    int admitted = 0, waiting = 0;
};

class Server {
public:
    enum State { WAITING = 0, ADMITTED = 1, REJECTED = 2, REMOVED = 3, FAILED = 4 };
    Server(int device, size_t budget_bytes);
    ~Server();
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    int add_session(SessionSpec spec);
    int state(int sid, std::string* why = nullptr);
    void remove_session(int sid);
    // Queue one matvec of session sid; den / val (complex64, the session's n
    // points) must stay valid until the request completes.
    long long submit(int sid, const std::complex<float>* den, std::complex<float>* val);
    // 0 done, 1 still pending after timeout_s; throws if the request failed.
    int wait(long long ticket, double timeout_s);
    int poll(long long ticket);  // 0 done, 1 pending, -1 failed
    ServerStats stats(bool reset);

private:
    struct Request {
        long long ticket;
        const std::complex<float>* den;
        std::complex<float>* val;
        double t_submit;
    };
    struct Entry {
        SessionSpec spec;
        State state = WAITING;
        std::string why;
        std::unique_ptr<Session> s;
        size_t bytes = 0;
        std::deque<Request> queue;
        float2* h_den = nullptr;  // pinned staging
        float2* h_val = nullptr;
        bool removing = false;
    };
    void admission_loop();
    void serving_loop();
    void rebuild();  // under mu_: the batch over the admitted sessions
    double now() const;

    int device_;
    size_t budget_;
    std::mutex mu_;
    std::condition_variable cv_work_, cv_admit_, cv_done_;
    bool stop_ = false;
    std::map<int, std::unique_ptr<Entry> > entries_;
    std::deque<int> waiting_;
    int next_sid_ = 0;
    long long next_ticket_ = 1;
    std::map<long long, int> done_;  // ticket -> 0 done / -1 failed (until read by wait/poll)
    std::map<long long, std::string> failures_;
    size_t used_ = 0;  // own device bytes of the admitted sessions (shared operator chunks apart)
    bool changed_ = false;        // admitted set changed since the batch was built
    bool blocked_ = false;        // the head of the waiting queue did not fit
    std::vector<int> slots_;      // batch instance -> sid
    std::vector<int> prev_tick_;  // sessions of the last tick
    std::unique_ptr<Batch> batch_;
    cudaStream_t stream_ = nullptr;
    int* d_active_ = nullptr;
    int* h_active_ = nullptr;
    std::vector<double> lat_ms_;
    long long ticks_ = 0, reqs_in_ticks_ = 0;
    double busy_s_ = 0;
    double last_tick_s_ = 0;  // duration of the last tick (sizes the gather window)
    std::thread admit_thread_, serve_thread_;
};

}  // namespace ddfmm
