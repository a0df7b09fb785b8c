// The partition server: a host thread that keeps a Scheduler (engine.cu)
// running while requests arrive.
//
// Continuous batching: a request is admitted as soon as the HBM budget and
// the active-job limit allow and joins the engine at its next tick, next to
// the jobs already on the device; a finished job leaves at the end of its
// tick and its arena goes back to the stream-ordered pool.  Each tick is one
// step (a merge step or a nodal sweep) of every active job, issued as
// multi-job launches, so requests that arrive while others run share the
// device with them instead of waiting for them.
#include "../../include/sbp.h"
#include "engine.h"
#include "job.h"

#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

struct sbp_server {
  sbp::Scheduler sch;
  sbp_server_options opt{};
  int device = 0;
  std::thread th;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<sbp::Run*> inbox;                                  // submitted, not yet queued
  std::unordered_map<int64_t, std::unique_ptr<sbp::Run>> live;  // every uncollected request
  int64_t next_id = 0;
  bool stop = false;
  sbp_status thread_status = SBP_OK;
  std::string thread_error;
  sbp_server_stats stats{};
  void loop();
};

namespace {

void finish_run(sbp::Run& r) {
  if (r.status == SBP_OK && r.R.status != 0) r.status = (sbp_status)r.R.status;
  r.R.status = r.status;
  r.R.ms_total = r.t_done_ms - r.t_admit_ms;
  r.finished = true;
}

}  // namespace

void sbp_server::loop() {
  cudaSetDevice(device);
  std::vector<sbp::Run*> done;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] { return stop || !inbox.empty() || !sch.idle(); });
      if (stop) {
        // cancel what has not reached the device
        for (sbp::Run* r : inbox) r->set_error(SBP_ERR_CANCELLED, "server stopped");
        for (size_t i = sch.queue_head; i < sch.queue.size(); ++i)
          sch.queue[i]->set_error(SBP_ERR_CANCELLED, "server stopped");
        for (sbp::Run* r : inbox) {
          r->t_done_ms = sbp::now_ms();
          finish_run(*r);
        }
        for (size_t i = sch.queue_head; i < sch.queue.size(); ++i) {
          sch.queue[i]->t_done_ms = sbp::now_ms();
          finish_run(*sch.queue[i]);
        }
        inbox.clear();
        sch.queue_head = sch.queue.size();
        cv_done.notify_all();
        if (sch.eng.runs.empty()) break;
      }
      while (!inbox.empty()) {
        sch.enqueue(inbox.front());
        inbox.pop_front();
      }
    }
    done.clear();
    sbp_status s = sch.step(done);
    std::lock_guard<std::mutex> lk(mu);
    if (s != SBP_OK) {
      // an engine failure ends every job on the device
      thread_status = s;
      thread_error = sbp_last_error();
      for (sbp::Run* r : sch.eng.runs) {
        r->set_error(s, thread_error);
        r->owned.reset();
        r->J = nullptr;
        r->t_done_ms = sbp::now_ms();
        done.push_back(r);
      }
      sch.eng.runs.clear();
      sch.used = 0.0;
    }
    for (sbp::Run* r : done) {
      finish_run(*r);
      ++stats.completed;
      if (r->status != SBP_OK) ++stats.failed;
    }
    stats.active = (int32_t)sch.eng.runs.size();
    stats.queued = (int32_t)(sch.queued() + inbox.size());
    stats.max_active_seen = sch.max_active_seen;
    stats.ticks = sch.eng.ticks;
    stats.bytes_active = sch.used;
    stats.peak_bytes = sch.peak;
    if (!done.empty()) cv_done.notify_all();
  }
}

using namespace sbp;

extern "C" {

void sbp_server_default_options(sbp_server_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  sbp_default_options(&o->partition);
}

sbp_status sbp_server_create(const sbp_server_options* o, sbp_server** out) {
  if (!o || !out) return fail(SBP_ERR_INVALID, "bad server arguments");
  *out = nullptr;
  sbp_status s = check_options(&o->partition);
  if (s != SBP_OK) return s;
  std::unique_ptr<sbp_server> h(new (std::nothrow) sbp_server());
  if (!h) return fail(SBP_ERR_NOMEM, "host allocation");
  h->opt = *o;
  h->device = resolve_device(o->partition.device);
  s = h->sch.init(h->device, o->hbm_budget, o->max_active);
  if (s != SBP_OK) return s;
  h->th = std::thread([p = h.get()] { p->loop(); });
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
                                         std::max(0, std::min(g->N, po.dense_max)));
  if (bytes > (double)srv->sch.budget)
    return fail(SBP_ERR_BUDGET, "job arena exceeds the HBM budget");
  std::unique_ptr<Run> r(new Run());
  r->graph_copy.assign(*g);
  r->graph_view = r->graph_copy.csr();
  r->graph = &r->graph_view;
  r->o = po;
  r->o.seed = seed;
  r->labels_store.assign((size_t)g->N, 0);
  r->labels_out = r->labels_store.data();
  r->t_submit_ms = now_ms();
  std::lock_guard<std::mutex> lk(srv->mu);
  if (srv->stop) return fail(SBP_ERR_CANCELLED, "server stopped");
  if (srv->opt.max_queued > 0 &&
      (int64_t)(srv->inbox.size() + srv->stats.queued) >= srv->opt.max_queued)
    return fail(SBP_ERR_BUSY, "request queue is full");
  r->id = srv->next_id++;
  *id = r->id;
  srv->inbox.push_back(r.get());
  srv->live[r->id] = std::move(r);
  ++srv->stats.submitted;
  srv->cv_work.notify_one();
  return SBP_OK;
}

sbp_status sbp_server_poll(sbp_server* srv, int64_t id, int32_t timeout_ms, int32_t* labels_out,
                           sbp_report* rep, sbp_job_times* times) {
  if (!srv) return fail(SBP_ERR_INVALID, "server is NULL");
  std::unique_lock<std::mutex> lk(srv->mu);
  auto it = srv->live.find(id);
  if (it == srv->live.end()) return fail(SBP_ERR_NOT_FOUND, "unknown request id");
  Run* r = it->second.get();
  if (!r->finished) {
    if (timeout_ms == 0) return fail(SBP_ERR_BUSY, "request still running");
    auto ready = [&] { return r->finished; };
    if (timeout_ms < 0) srv->cv_done.wait(lk, ready);
    else if (!srv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
      return fail(SBP_ERR_BUSY, "request still running");
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
  srv->live.erase(it);
  if (st != SBP_OK) return fail(st, msg);
  return SBP_OK;
}

sbp_status sbp_server_stats_get(sbp_server* srv, sbp_server_stats* out) {
  if (!srv || !out) return fail(SBP_ERR_INVALID, "bad arguments");
  std::lock_guard<std::mutex> lk(srv->mu);
  *out = srv->stats;
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
  if (srv->th.joinable()) srv->th.join();
  delete srv;
  return SBP_OK;
}

}  // extern "C"
