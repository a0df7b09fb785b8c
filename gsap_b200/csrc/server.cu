// The partition server: host threads that keep Schedulers (engine.cu)
// running while requests arrive.
//
// Continuous batching: a request is admitted as soon as the HBM budget and
// the active-job limit allow and joins its lane's engine at the next tick,
// next to the jobs already on the device; a finished job leaves at the end
// of its tick and its arena goes back to the stream-ordered pool.  Each tick
// is one step (a merge step or queued nodal sweeps) of every active job of
// the lane, issued as multi-job launches.
//
// Lanes: a tick lasts as long as its largest job's step, so requests are
// split by graph size into lanes, each with its own engine, stream and host
// thread, all drawing on one HBM budget.  The GPU runs the lanes' launches
// side by side, and a small request's steps do not wait for a large one's.
#include "../../include/sbp.h"
#include "engine.h"
#include "job.h"

#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

namespace {

struct Lane {
  sbp::Scheduler sch;
  std::thread th;
  std::deque<sbp::Run*> inbox;  // submitted to this lane, not yet queued
  int32_t active = 0, queued = 0, max_active_seen = 0;
  int64_t ticks = 0;
};

}  // namespace

struct sbp_server {
  sbp_server_options opt{};
  int device = 0;
  int32_t split = 10000;
  std::shared_ptr<sbp::HbmBudget> hbm;
  std::vector<std::unique_ptr<Lane>> lanes;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::unordered_map<int64_t, std::unique_ptr<sbp::Run>> live;  // every uncollected request
  int64_t next_id = 0;
  bool stop = false;
  sbp_status thread_status = SBP_OK;
  std::string thread_error;
  int64_t completed = 0, failed = 0, submitted = 0;
  void loop(Lane& L);
  int32_t queued_total() const {
    int32_t q = 0;
    for (const auto& l : lanes) q += l->queued + (int32_t)l->inbox.size();
    return q;
  }
};

namespace {

void finish_run(sbp::Run& r) {
  if (r.status == SBP_OK && r.R.status != 0) r.status = (sbp_status)r.R.status;
  r.R.status = r.status;
  r.R.ms_total = r.t_done_ms - r.t_admit_ms;
  r.finished = true;
}

}  // namespace

void sbp_server::loop(Lane& L) {
  cudaSetDevice(device);
  sbp::Scheduler& sch = L.sch;
  std::vector<sbp::Run*> done;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] { return stop || !L.inbox.empty() || !sch.idle(); });
      if (stop) {
        // cancel what has not reached the device
        const double t = sbp::now_ms();
        for (sbp::Run* r : L.inbox) {
          r->set_error(SBP_ERR_CANCELLED, "server stopped");
          r->t_done_ms = t;
          finish_run(*r);
        }
        for (size_t i = sch.queue_head; i < sch.queue.size(); ++i) {
          sch.queue[i]->set_error(SBP_ERR_CANCELLED, "server stopped");
          sch.queue[i]->t_done_ms = t;
          finish_run(*sch.queue[i]);
        }
        L.inbox.clear();
        sch.queue_head = sch.queue.size();
        cv_done.notify_all();
        if (sch.eng.runs.empty()) break;
      }
      while (!L.inbox.empty()) {
        sch.enqueue(L.inbox.front());
        L.inbox.pop_front();
      }
    }
    done.clear();
    sbp_status s = sch.step(done);
    std::lock_guard<std::mutex> lk(mu);
    if (s != SBP_OK) {
      // an engine failure ends every job of the lane that is on the device
      thread_status = s;
      thread_error = sbp_last_error();
      std::lock_guard<std::mutex> submit(sbp::cuda_submit_mutex());
      for (sbp::Run* r : sch.eng.runs) {
        r->set_error(s, thread_error);
        sch.hbm->give(r->admit_bytes);
        r->owned.reset();
        r->J = nullptr;
        r->release_events();
        r->t_done_ms = sbp::now_ms();
        done.push_back(r);
      }
      sch.eng.runs.clear();
    }
    for (sbp::Run* r : done) {
      finish_run(*r);
      ++completed;
      if (r->status != SBP_OK) ++failed;
    }
    L.active = (int32_t)sch.eng.runs.size();
    L.queued = (int32_t)sch.queued();
    L.max_active_seen = sch.max_active_seen;
    L.ticks = sch.eng.ticks;
    if (!done.empty()) cv_done.notify_all();
  }
}

using namespace sbp;

extern "C" {

void sbp_server_default_options(sbp_server_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  sbp_default_options(&o->partition);
  o->lanes = 2;
  o->lane_split = 10000;
}

sbp_status sbp_server_create(const sbp_server_options* o, sbp_server** out) {
  if (!o || !out) return fail(SBP_ERR_INVALID, "bad server arguments");
  *out = nullptr;
  sbp_status s = check_options(&o->partition);
  if (s != SBP_OK) return s;
  if (o->lanes < 0 || o->lanes > 8) return fail(SBP_ERR_INVALID, "lanes must be in [0, 8]");
  std::unique_ptr<sbp_server> h(new (std::nothrow) sbp_server());
  if (!h) return fail(SBP_ERR_NOMEM, "host allocation");
  h->opt = *o;
  h->device = resolve_device(o->partition.device);
  h->split = o->lane_split > 0 ? o->lane_split : 10000;
  const int nl = o->lanes > 0 ? o->lanes : 2;
  for (int i = 0; i < nl; ++i) {
    h->lanes.emplace_back(new Lane());
    s = h->lanes.back()->sch.init(h->device, o->hbm_budget, o->max_active, h->hbm);
    if (s != SBP_OK) return s;
    if (!h->hbm) h->hbm = h->lanes.back()->sch.hbm;
  }
  for (auto& l : h->lanes) {
    Lane* lp = l.get();
    l->th = std::thread([p = h.get(), lp] { p->loop(*lp); });
  }
  *out = h.release();
  return SBP_OK;
}

sbp_status sbp_server_submit(sbp_server* srv, const sbp_graph_csr* g, uint64_t seed,
                             int64_t* id) {
  if (!srv || !id) return fail(SBP_ERR_INVALID, "bad submit arguments");
  sbp_status s = validate_graph(g);
  if (s != SBP_OK) return s;
  const sbp_options& po = srv->opt.partition;
  const double bytes = (double)job_bytes(g->N, g->E, po.num_proposals, po.max_nodal_itr,
                                         dense_limit(g->N, g->E, po.dense_max));
  if (bytes > srv->hbm->cap) return fail(SBP_ERR_BUDGET, "job arena exceeds the HBM budget");
  std::unique_ptr<Run> r(new Run());
  r->graph_copy.assign(*g);
  r->graph_view = r->graph_copy.csr();
  r->graph = &r->graph_view;
  r->o = po;
  r->o.seed = seed;
  r->labels_store.assign((size_t)g->N, 0);
  r->labels_out = r->labels_store.data();
  r->t_submit_ms = now_ms();
  // lane 0 takes the smallest graphs, each further lane sizes up to 4x more
  size_t lane = 0;
  for (int64_t lim = srv->split; lane + 1 < srv->lanes.size() && g->N > lim; lim *= 4) ++lane;
  std::lock_guard<std::mutex> lk(srv->mu);
  if (srv->stop) return fail(SBP_ERR_CANCELLED, "server stopped");
  if (srv->opt.max_queued > 0 && srv->queued_total() >= srv->opt.max_queued)
    return fail(SBP_ERR_BUSY, "request queue is full");
  r->id = srv->next_id++;
  *id = r->id;
  srv->lanes[lane]->inbox.push_back(r.get());
  srv->live[r->id] = std::move(r);
  ++srv->submitted;
  srv->cv_work.notify_all();
  return SBP_OK;
}

sbp_status sbp_server_poll(sbp_server* srv, int64_t id, int32_t timeout_ms, int32_t* labels_out,
                           sbp_report* rep, sbp_job_times* times) {
  if (!srv) return fail(SBP_ERR_INVALID, "server is NULL");
  std::unique_lock<std::mutex> lk(srv->mu);
  // Another thread polling the same id may collect (and free) the request
  // while this one waits, so the request is looked up afresh after every
  // wake-up and never held across the wait.
  auto lookup = [&]() -> Run* {
    auto it = srv->live.find(id);
    return it == srv->live.end() ? nullptr : it->second.get();
  };
  Run* r = lookup();
  if (!r) return fail(SBP_ERR_NOT_FOUND, "unknown request id");
  if (!r->finished) {
    if (timeout_ms == 0) return fail(SBP_ERR_BUSY, "request still running");
    auto ready = [&] {
      Run* q = lookup();
      return !q || q->finished;
    };
    if (timeout_ms < 0) srv->cv_done.wait(lk, ready);
    else if (!srv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
      return fail(SBP_ERR_BUSY, "request still running");
    r = lookup();
    if (!r) return fail(SBP_ERR_NOT_FOUND, "request collected by another poll");
  }
  if (labels_out) std::memcpy(labels_out, r->labels_store.data(), 4 * r->labels_store.size());
  if (rep) *rep = r->R;
  if (times) {
    const double admit = r->t_admit_ms > 0.0 ? r->t_admit_ms : r->t_done_ms;
    times->ms_queue = admit - r->t_submit_ms;
    times->ms_run = r->t_done_ms - admit;
    times->ms_latency = r->t_done_ms - r->t_submit_ms;
  }
  const sbp_status st = r->status;
  const std::string msg = r->error;
  srv->live.erase(id);
  // a second poller of this id waits on cv_done: wake it to see it gone
  srv->cv_done.notify_all();
  if (st != SBP_OK) return fail(st, msg);
  return SBP_OK;
}

sbp_status sbp_server_stats_get(sbp_server* srv, sbp_server_stats* out) {
  if (!srv || !out) return fail(SBP_ERR_INVALID, "bad arguments");
  std::lock_guard<std::mutex> lk(srv->mu);
  std::memset(out, 0, sizeof(*out));
  out->submitted = srv->submitted;
  out->completed = srv->completed;
  out->failed = srv->failed;
  for (const auto& l : srv->lanes) {
    out->active += l->active;
    out->queued += l->queued + (int32_t)l->inbox.size();
    out->max_active_seen += l->max_active_seen;
    out->ticks += l->ticks;
  }
  {
    std::lock_guard<std::mutex> lb(srv->hbm->mu);
    out->bytes_active = srv->hbm->used;
    out->peak_bytes = srv->hbm->peak;
  }
  if (srv->thread_status != SBP_OK) return fail(srv->thread_status, srv->thread_error);
  return SBP_OK;
}

sbp_status sbp_server_destroy(sbp_server* srv) {
  if (!srv) return SBP_OK;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->stop = true;
  }
  srv->cv_work.notify_all();
  for (auto& l : srv->lanes)
    if (l->th.joinable()) l->th.join();
  delete srv;
  return SBP_OK;
}

}  // extern "C"
