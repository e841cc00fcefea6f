// Serving form: a device-resident request loop with continuous batching.
//
// The reference runs one query at a time in the calling thread
// (execution/executable_query.cc:199-255).  A server here owns N slots; each
// slot is a Context with its own CUDA stream that shares the parent's
// HBM-resident tables, enum dictionaries and compiled pipelines, and a worker
// thread.  Requests queue on arrival; a free slot admits the oldest request
// whose estimated HBM footprint fits the remaining budget (requests that
// arrive while others run are admitted as soon as a slot and memory free up),
// so the kernels of several queries overlap on the device.  Each request's
// latency runs from submission to completion; the server reports p50/p99 and
// throughput.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <sstream>
#include <thread>

#include "capi_internal.h"

namespace kdb {
namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t id;
  std::string plan;
  int64_t footprint;
  Clock::time_point submitted;
  Clock::time_point started, finished;
  int status = 1;  // 1 = pending, 0 = done, < 0 = error code
  std::string error;
  HostResult result;
};

// Bytes of device memory a plan will hold at its peak, estimated from the
// base columns it scans: materialised intermediates and tables are at most a
// few times the bytes read.
int64_t EstimateFootprint(const Context& ctx, const plan::Operator& op) {
  int64_t b = 0;
  if (op.kind == plan::OpKind::SCAN || op.kind == plan::OpKind::SCAN_SELECT) {
    auto it = ctx.tables.find(op.relation);
    if (it != ctx.tables.end())
      for (const auto& sc : op.scan_columns) {
        auto c = it->second.cols.find(sc.name);
        if (c != it->second.cols.end()) b += static_cast<int64_t>(c->second.bytes);
      }
    return 2 * b;
  }
  for (const auto& c : op.children) b += EstimateFootprint(ctx, *c);
  return b;
}

}  // namespace

class Server {
 public:
  Server(Context& parent, int slots, int64_t hbm_budget) : budget_(hbm_budget) {
    // Build state kept across requests (Skinner children and their join
    // indexes) takes up to a quarter of the budget; requests are admitted
    // against the rest.
    cache_ = MakeBuildCache(static_cast<size_t>(hbm_budget / 4));
    budget_ = hbm_budget - hbm_budget / 4;
    for (int i = 0; i < slots; i++) {
      slots_.push_back(std::make_unique<Context>(parent));
      slots_.back()->ReserveHostBlocks(4, 16 << 20);  // pinned result blocks up front: no host-alloc syncs later
      slots_.back()->build_cache = cache_;
    }
    for (int i = 0; i < slots; i++) workers_.emplace_back([this, i] { Loop(i); });
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> lock(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
    // cached entries free their memory on the streams of the slots that
    // built them: release them while those slots still exist
    for (auto& s : slots_) s->build_cache.reset();
    cache_.reset();
  }

  int64_t Submit(const std::string& plan_json, const Context& catalog) {
    auto plan = plan::ParsePlan(plan_json);  // reject bad plans at submission
    auto r = std::make_shared<Request>();
    r->plan = plan_json;
    r->footprint = std::min(EstimateFootprint(catalog, *plan), budget_);
    r->submitted = Clock::now();
    std::lock_guard<std::mutex> lock(mu_);
    r->id = next_id_++;
    queue_.push_back(r);
    all_[r->id] = r;
    cv_.notify_one();
    return r->id;
  }

  // 1 pending, 0 done, < 0 error; blocks up to timeout_ms when wait is set.
  int Poll(int64_t id, int64_t timeout_ms, std::shared_ptr<Request>* out) {
    std::unique_lock<std::mutex> lock(mu_);
    auto it = all_.find(id);
    if (it == all_.end()) return KDB_ERR_INVALID;
    auto r = it->second;
    if (timeout_ms > 0)
      done_cv_.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] { return r->status != 1; });
    if (out) *out = r;
    return r->status;
  }

  void Forget(int64_t id) {
    std::lock_guard<std::mutex> lock(mu_);
    all_.erase(id);
  }

  std::string Stats() {
    std::lock_guard<std::mutex> lock(mu_);
    std::vector<double> lat = lat_ms_, svc = svc_ms_;
    int64_t done = static_cast<int64_t>(lat.size()), failed = failed_;
    std::sort(lat.begin(), lat.end());
    std::sort(svc.begin(), svc.end());
    auto pct = [](const std::vector<double>& v, double p) {
      if (v.empty()) return 0.0;
      size_t i = static_cast<size_t>(p * (v.size() - 1) + 0.5);
      return v[std::min(i, v.size() - 1)];
    };
    double span = done ? std::chrono::duration<double>(last_finish_ - first_submit_).count() : 0;
    std::ostringstream o;
    o << "{\"completed\":" << done << ",\"failed\":" << failed << ",\"p50_ms\":" << pct(lat, 0.5)
      << ",\"p99_ms\":" << pct(lat, 0.99) << ",\"max_ms\":" << (lat.empty() ? 0 : lat.back())
      << ",\"service_p50_ms\":" << pct(svc, 0.5) << ",\"queries_per_second\":" << (span > 0 ? done / span : 0)
      << ",\"peak_in_flight\":" << peak_in_flight_ << ",\"slots\":" << slots_.size()
      << ",\"hbm_budget\":" << budget_ << ",\"kernel_launches\":" << launches_;
    int64_t hits = 0, misses = 0, bytes = 0, entries = 0;
    if (cache_) BuildCacheStats(*cache_, &hits, &misses, &bytes, &entries);
    o << ",\"build_cache_hits\":" << hits << ",\"build_cache_misses\":" << misses
      << ",\"build_cache_bytes\":" << bytes << ",\"build_cache_entries\":" << entries << "}";
    return o.str();
  }

 private:
  void Loop(int slot) {
    Context& ctx = *slots_[slot];
    cudaSetDevice(ctx.device);
    while (true) {
      std::shared_ptr<Request> r;
      {
        std::unique_lock<std::mutex> lock(mu_);
        cv_.wait(lock, [&] { return stop_ || Admissible() >= 0; });
        if (stop_) return;
        size_t i = static_cast<size_t>(Admissible());
        r = queue_[i];
        queue_.erase(queue_.begin() + static_cast<std::ptrdiff_t>(i));
        in_use_ += r->footprint;
        in_flight_++;
        peak_in_flight_ = std::max(peak_in_flight_, in_flight_);
        r->started = Clock::now();
      }
      int status = 0;
      std::string err;
      HostResult res;
      const int64_t launches0 = ctx.kernel_launches;
      try {
        auto plan = plan::ParsePlan(r->plan);
        res = ExecutePlan(ctx, *plan);
      } catch (const Error& e) {
        status = e.code;
        err = e.what();
      } catch (const std::exception& e) {
        status = KDB_ERR_INVALID;
        err = e.what();
      }
      {
        std::lock_guard<std::mutex> lock(mu_);
        r->finished = Clock::now();
        r->result = std::move(res);
        r->error = err;
        r->status = status;
        in_use_ -= r->footprint;
        in_flight_--;
        launches_ += ctx.kernel_launches - launches0;
        if (status == 0) {
          lat_ms_.push_back(std::chrono::duration<double, std::milli>(r->finished - r->submitted).count());
          svc_ms_.push_back(std::chrono::duration<double, std::milli>(r->finished - r->started).count());
          if (lat_ms_.size() == 1 || r->submitted < first_submit_) first_submit_ = r->submitted;
          if (lat_ms_.size() == 1 || r->finished > last_finish_) last_finish_ = r->finished;
        } else {
          failed_++;
        }
      }
      done_cv_.notify_all();
      cv_.notify_all();  // freed memory may admit a queued request
    }
  }

  // Oldest queued request that fits the free budget (-1 if none).
  long Admissible() const {
    for (size_t i = 0; i < queue_.size(); i++)
      if (in_use_ + queue_[i]->footprint <= budget_ || in_flight_ == 0) return static_cast<long>(i);
    return -1;
  }

  int64_t budget_;
  std::shared_ptr<BuildCache> cache_;
  std::vector<std::unique_ptr<Context>> slots_;
  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  std::deque<std::shared_ptr<Request>> queue_;
  std::map<int64_t, std::shared_ptr<Request>> all_;
  int64_t next_id_ = 1;
  int64_t in_use_ = 0;
  int in_flight_ = 0, peak_in_flight_ = 0;
  bool stop_ = false;
  std::vector<double> lat_ms_, svc_ms_;  // completed requests
  int64_t failed_ = 0;
  int64_t launches_ = 0;  // kernels launched by all completed requests
  Clock::time_point first_submit_, last_finish_;
};

}  // namespace kdb

struct kdb_server {
  kdb_ctx* owner;
  std::unique_ptr<kdb::Server> s;
};

extern "C" {

int kdb_server_start(kdb_ctx* ctx, int32_t slots, int64_t hbm_budget_bytes, kdb_server** out) {
  if (!ctx || !out || slots < 1 || slots > 64 || hbm_budget_bytes <= 0) return KDB_ERR_INVALID;
  *out = nullptr;
  try {
    kdb::Context& c = *kdb_ctx_context(ctx);
    if (c.dry) throw kdb::Error(KDB_ERR_UNSUPPORTED, "serving needs a GPU context");
    auto s = std::make_unique<kdb_server>();
    s->owner = ctx;
    s->s = std::make_unique<kdb::Server>(c, slots, hbm_budget_bytes);
    *out = s.release();
    return KDB_OK;
  } catch (const kdb::Error& e) {
    kdb_ctx_set_error(ctx, e.what());
    return e.code;
  } catch (const std::exception& e) {
    kdb_ctx_set_error(ctx, e.what());
    return KDB_ERR_CUDA;
  }
}

int64_t kdb_server_submit(kdb_server* s, const char* plan_json) {
  if (!s || !plan_json) return KDB_ERR_INVALID;
  try {
    return s->s->Submit(plan_json, *kdb_ctx_context(s->owner));
  } catch (const std::exception& e) {
    kdb_ctx_set_error(s->owner, e.what());
    return KDB_ERR_INVALID;
  }
}

int kdb_server_poll(kdb_server* s, int64_t ticket, int64_t wait_ms, kdb_result** out) {
  if (!s) return KDB_ERR_INVALID;
  if (out) *out = nullptr;
  std::shared_ptr<kdb::Request> r;
  int st = s->s->Poll(ticket, wait_ms, &r);
  if (st == 0 && out) {
    auto res = std::make_unique<kdb_result>();
    res->r = r->result;
    *out = res.release();
    s->s->Forget(ticket);
  } else if (st < 0 && r) {
    kdb_ctx_set_error(s->owner, r->error);
    s->s->Forget(ticket);
  }
  return st;
}

int64_t kdb_server_stats(kdb_server* s, char* buf, int64_t cap) {
  if (!s) return KDB_ERR_INVALID;
  std::string j = s->s->Stats();
  if (buf && cap > 0) {
    int64_t n = std::min<int64_t>(cap - 1, j.size());
    std::memcpy(buf, j.data(), n);
    buf[n] = 0;
  }
  return static_cast<int64_t>(j.size()) + 1;
}

void kdb_server_stop(kdb_server* s) { delete s; }

}  // extern "C"
