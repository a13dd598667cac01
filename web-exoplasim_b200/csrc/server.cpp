// The batched server of the C ABI (exogcm_server_*): continuous batching of
// many planet runs on one GPU, above the engine calls. It has no counterpart
// file in the reference, whose page runs one planet per worker
// (runner/webgpu/gcm.worker.ts); it serves many such runs at once the way
// the worker steps one: batches of steps submitted asynchronously
// (exogcm_step_async, the worker's IN_FLIGHT batches), a run stopped exactly
// at its last step, and the reference's instability failure.
//
// Runs of one resolution (T, L) share engines ("blocks" of slots). Every
// resolution draws on one device-byte budget by its per-slot footprint:
// a request is admitted into a free slot of its resolution, or into a new
// block when the budget has room, made if need be by destroying empty blocks
// of other resolutions. One exogcm_server_pump call submits every block that
// has running slots, admits queued requests while those batches run (their
// host set-up overlaps the device work), waits for the batches and collects
// the runs that finished (their spectral prognostic fields are kept for
// exogcm_server_result) or became unstable.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/exogcm.h"
#include "fields.h"

namespace exogcm {
void set_error(const std::string& message);  // engine.cu
}

struct exogcm_server;

namespace {

struct Failure : std::runtime_error {
  int code;
  Failure(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// An engine call's status; its message is already the library's last error.
void call(int status, const char* what) {
  if (status == EXOGCM_OK) return;
  char buf[512];
  exogcm_last_error(buf, sizeof(buf));
  throw Failure(status, std::string(what) + ": " + buf);
}

int nlat_of(int truncation) { return truncation == 21 ? 32 : truncation == 42 ? 64 : 96; }

const char* const kResultFields[] = {"st", "sz", "sd", "sq", "sp"};

struct Request {
  long id = 0;
  exogcm_planet planet{};
  // owned copies of the boundary arrays
  std::vector<double> mask, oro, sst, ice, t, q;
  int sst_months = 0, ice_months = 0;
  bool has_oro = false;
  long steps = 0;
  int status = EXOGCM_REQUEST_QUEUED;
  long steps_done = 0;
  long start_step = 0;
  std::map<std::string, std::vector<float>> result;

  exogcm_boundary boundary() const {
    exogcm_boundary b{};
    b.land_mask = mask.data();
    b.orography = has_oro ? oro.data() : nullptr;
    b.sst = sst.empty() ? nullptr : sst.data();
    b.sst_months = sst_months;
    b.ice_cover = ice.empty() ? nullptr : ice.data();
    b.ice_cover_months = ice_months;
    b.t_init = t.data();
    b.q_init = q.data();
    return b;
  }
};

struct Block {
  int truncation, levels, slots;
  exogcm_engine* engine = nullptr;
  std::vector<long> running;  // request id per slot, 0 when free
  std::vector<long> stop;     // model step at which the slot's run ends
  bool in_flight = false;

  int free_slot() const {
    for (int s = 0; s < slots; ++s)
      if (!running[s]) return s;
    return -1;
  }
  int busy() const {
    int n = 0;
    for (long r : running) n += r ? 1 : 0;
    return n;
  }
};

}  // namespace

struct exogcm_server {
  exogcm_server_options opt{};
  long next_id = 1;
  std::deque<long> queue;                       // requests waiting for a slot, oldest first
  std::map<long, std::unique_ptr<Request>> requests;
  std::vector<std::unique_ptr<Block>> blocks;
  std::map<std::pair<int, int>, double> slot_bytes;  // per (T, L)

  ~exogcm_server() {
    for (auto& b : blocks) {
      if (b->in_flight) exogcm_wait(b->engine);
      exogcm_destroy(b->engine);
    }
  }

  // Device bytes one slot of a (T, L) engine holds: every state field of
  // the layout (fields.h), counted on a one-slot engine once, and its
  // per-slot tables.
  double bytes_per_slot(int T, int L) {
    const auto key = std::make_pair(T, L);
    auto it = slot_bytes.find(key);
    if (it != slot_bytes.end()) return it->second;
    exogcm_engine* probe = nullptr;
    call(exogcm_create(T, L, 1, opt.mode, &probe), "server: engine");
    size_t total = 0;
#define EXOGCM_SERVER_FIELD(name, shape, count) #name,
    static const char* const names[] = {EXOGCM_FIELDS(EXOGCM_SERVER_FIELD)};
#undef EXOGCM_SERVER_FIELD
    for (const char* name : names) {
      size_t n = 0;
      const int status = exogcm_field_size(probe, name, &n);
      if (status != EXOGCM_OK) {
        exogcm_destroy(probe);
        call(status, "server: field size");
      }
      total += n;
    }
    exogcm_destroy(probe);
    const double bytes = (double)total * sizeof(float) + 64 * 1024;
    slot_bytes[key] = bytes;
    return bytes;
  }

  // Slots of a new block: `block_slots` at T21 L5, fewer at larger
  // resolutions so a block's bytes stay about the same.
  int block_slots_for(int T, int L) {
    const double ratio = bytes_per_slot(21, 5) / bytes_per_slot(T, L);
    return std::max(1, (int)std::lround(opt.block_slots * std::min(1.0, 4.0 * ratio)));
  }

  double used_bytes() {
    double used = 0;
    for (auto& b : blocks) used += b->slots * bytes_per_slot(b->truncation, b->levels);
    return used;
  }

  Block* free_block(int T, int L) {
    for (auto& b : blocks)
      if (b->truncation == T && b->levels == L && b->free_slot() >= 0) return b.get();
    return nullptr;
  }

  // A new block for (T, L) within the budget, destroying empty blocks of
  // other resolutions for room; nullptr when there is none.
  Block* grow(int T, int L) {
    const int n = block_slots_for(T, L);
    const double need = n * bytes_per_slot(T, L);
    if (need > opt.budget_bytes) return nullptr;
    while (used_bytes() + need > opt.budget_bytes) {
      auto it = std::find_if(blocks.begin(), blocks.end(), [&](const std::unique_ptr<Block>& b) {
        return b->busy() == 0 && !(b->truncation == T && b->levels == L);
      });
      if (it == blocks.end()) return nullptr;
      if ((*it)->in_flight) exogcm_wait((*it)->engine);
      exogcm_destroy((*it)->engine);
      blocks.erase(it);
    }
    auto b = std::make_unique<Block>();
    b->truncation = T;
    b->levels = L;
    b->slots = n;
    b->running.assign(n, 0);
    b->stop.assign(n, 0);
    const int status = exogcm_create(T, L, n, opt.mode, &b->engine);
    if (status == EXOGCM_ENOMEM) return nullptr;  // the device has less room than the budget says
    call(status, "server: block");
    blocks.push_back(std::move(b));
    return blocks.back().get();
  }

  void admit() {
    std::deque<long> waiting;
    while (!queue.empty()) {
      const long id = queue.front();
      queue.pop_front();
      Request& r = *requests.at(id);
      const int T = r.planet.truncation, L = r.planet.levels;
      if (block_slots_for(T, L) * bytes_per_slot(T, L) > opt.budget_bytes) {
        r.status = EXOGCM_REQUEST_REJECTED;
        continue;
      }
      Block* b = free_block(T, L);
      if (!b) b = grow(T, L);
      if (!b) {
        waiting.push_back(id);
        continue;
      }
      const int slot = b->free_slot();
      const exogcm_boundary bd = r.boundary();
      const int status = exogcm_configure(b->engine, slot, &r.planet, &bd);
      if (status != EXOGCM_OK) {  // the planet's set-up is invalid (the message is the last error)
        r.status = EXOGCM_REQUEST_FAILED;
        continue;
      }
      long step = 0;
      int left = 0, active = 0;
      call(exogcm_slot_info(b->engine, slot, &step, &left, &active), "server: slot");
      r.start_step = step;
      b->stop[slot] = step + r.steps;
      call(exogcm_set_stop(b->engine, slot, b->stop[slot]), "server: stop");
      b->running[slot] = id;
      r.status = EXOGCM_REQUEST_RUNNING;
    }
    queue = std::move(waiting);
  }

  void collect(Block& b) {
    std::vector<int> flags(b.slots, 0);
    call(exogcm_unstable(b.engine, flags.data(), b.slots), "server: stability");
    for (int s = 0; s < b.slots; ++s) {
      if (!b.running[s]) continue;
      Request& r = *requests.at(b.running[s]);
      long step = 0;
      int left = 0, active = 0;
      call(exogcm_slot_info(b.engine, s, &step, &left, &active), "server: slot");
      r.steps_done = std::max(0L, step - r.start_step);
      const bool failed = flags[s] != 0;
      if (!failed && !(left == 0 && step >= b.stop[s])) continue;
      if (failed) {
        r.status = EXOGCM_REQUEST_FAILED;
      } else {
        for (const char* name : kResultFields) {
          size_t n = 0;
          call(exogcm_field_size(b.engine, name, &n), "server: result");
          std::vector<float> v(n);
          call(exogcm_read_field(b.engine, s, name, v.data(), n), "server: result");
          r.result[name] = std::move(v);
        }
        r.status = EXOGCM_REQUEST_FINISHED;
      }
      call(exogcm_release(b.engine, s), "server: release");
      b.running[s] = 0;
    }
  }

  void pump() {
    for (auto& b : blocks)
      if (b->busy()) {
        call(exogcm_step_async(b->engine, opt.chunk_steps, 1 << 30), "server: step");
        b->in_flight = true;
      }
    admit();  // queued requests are set up while the submitted batches run
    for (auto& b : blocks)
      if (b->in_flight) {
        b->in_flight = false;
        call(exogcm_wait(b->engine), "server: wait");
      }
    for (auto& b : blocks)
      if (b->busy()) collect(*b);
  }
};

namespace {

template <typename F>
int server_guard(F&& f) {
  try {
    f();
    return EXOGCM_OK;
  } catch (const Failure& e) {
    exogcm::set_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    exogcm::set_error("server: host allocation failed");
    return EXOGCM_ENOMEM;
  } catch (const std::exception& e) {
    exogcm::set_error(std::string("server: ") + e.what());
    return EXOGCM_EINVAL;
  }
}

Request& find(exogcm_server* s, long id) {
  auto it = s->requests.find(id);
  if (it == s->requests.end()) throw Failure(EXOGCM_EINVAL, "server: no request " + std::to_string(id));
  return *it->second;
}

}  // namespace

extern "C" {

int exogcm_server_create(const exogcm_server_options* options, exogcm_server** out) {
  return server_guard([&] {
    if (!options || !out) throw Failure(EXOGCM_EINVAL, "server: null argument");
    *out = nullptr;
    if (!(options->budget_bytes > 0) || options->block_slots < 1 || options->block_slots > 4096 ||
        options->chunk_steps < 1 || options->chunk_steps > 64 || options->mode < 0 || options->mode > 2)
      throw Failure(EXOGCM_EINVAL,
                    "server: budget must be positive, block_slots 1..4096, chunk_steps 1..64, mode 0..2");
    auto s = std::make_unique<exogcm_server>();
    s->opt = *options;
    *out = s.release();
  });
}

void exogcm_server_destroy(exogcm_server* server) { delete server; }

int exogcm_server_submit(exogcm_server* s, const exogcm_planet* planet, const exogcm_boundary* boundary, long steps,
                         long* request) {
  return server_guard([&] {
    if (!s || !planet || !boundary || !request) throw Failure(EXOGCM_EINVAL, "server: null argument");
    if (steps < 1) throw Failure(EXOGCM_EINVAL, "server: a run needs at least one step");
    const int T = planet->truncation, L = planet->levels;
    if ((T != 21 && T != 42 && T != 63) || (L != 5 && L != 10))
      throw Failure(EXOGCM_EINVAL, "server: truncation must be 21, 42 or 63 and levels 5 or 10");
    if (!boundary->land_mask || !boundary->t_init || !boundary->q_init)
      throw Failure(EXOGCM_EINVAL, "server: land mask and initial fields required");
    const size_t nhor = 2 * (size_t)nlat_of(T) * nlat_of(T);
    auto r = std::make_unique<Request>();
    r->id = s->next_id++;
    r->planet = *planet;
    r->steps = steps;
    r->mask.assign(boundary->land_mask, boundary->land_mask + nhor);
    if (boundary->orography) {
      r->has_oro = true;
      r->oro.assign(boundary->orography, boundary->orography + nhor);
    }
    if (boundary->sst && boundary->sst_months > 0) {
      r->sst_months = boundary->sst_months;
      r->sst.assign(boundary->sst, boundary->sst + nhor * boundary->sst_months);
    }
    if (boundary->ice_cover && boundary->ice_cover_months > 0) {
      r->ice_months = boundary->ice_cover_months;
      r->ice.assign(boundary->ice_cover, boundary->ice_cover + nhor * boundary->ice_cover_months);
    }
    r->t.assign(boundary->t_init, boundary->t_init + nhor * L);
    r->q.assign(boundary->q_init, boundary->q_init + nhor * L);
    *request = r->id;
    s->queue.push_back(r->id);
    s->requests[r->id] = std::move(r);
  });
}

int exogcm_server_pump(exogcm_server* s, int* active) {
  return server_guard([&] {
    if (!s) throw Failure(EXOGCM_EINVAL, "server: null server");
    s->pump();
    if (active) {
      int n = 0;
      for (auto& kv : s->requests)
        n += kv.second->status == EXOGCM_REQUEST_QUEUED || kv.second->status == EXOGCM_REQUEST_RUNNING;
      *active = n;
    }
  });
}

int exogcm_server_poll(exogcm_server* s, long request, int* status, long* steps_done) {
  return server_guard([&] {
    if (!s || !status) throw Failure(EXOGCM_EINVAL, "server: null argument");
    const Request& r = find(s, request);
    *status = r.status;
    if (steps_done) *steps_done = r.steps_done;
  });
}

int exogcm_server_result(exogcm_server* s, long request, const char* field, float* values, size_t count) {
  return server_guard([&] {
    if (!s || !field) throw Failure(EXOGCM_EINVAL, "server: null argument");
    const Request& r = find(s, request);
    if (r.status != EXOGCM_REQUEST_FINISHED) throw Failure(EXOGCM_ESTATE, "server: the run has not finished");
    auto it = r.result.find(field);
    if (it == r.result.end())
      throw Failure(EXOGCM_EINVAL, std::string("server: no result field ") + field + " (st, sz, sd, sq, sp)");
    if (!values || count != it->second.size())
      throw Failure(EXOGCM_EINVAL, "server: result buffer must hold " + std::to_string(it->second.size()) + " values");
    std::memcpy(values, it->second.data(), count * sizeof(float));
  });
}

int exogcm_server_release(exogcm_server* s, long request) {
  return server_guard([&] {
    if (!s) throw Failure(EXOGCM_EINVAL, "server: null server");
    Request& r = find(s, request);
    if (r.status == EXOGCM_REQUEST_QUEUED || r.status == EXOGCM_REQUEST_RUNNING)
      throw Failure(EXOGCM_ESTATE, "server: the run is still queued or running");
    s->requests.erase(request);
  });
}

}  // extern "C"
