// nbs2.cpp -- NBS2 trajectory writer (the format of src/Main.cpp:13-49,
// read by load_sim.py).  Plain host code behind the C ABI.
#include "nbx.h"

#include <cstdio>
#include <vector>

struct nbx_nbs2 {
  std::FILE *f = nullptr;
  uint32_t n = 0;
  uint32_t completed = 0;
  std::vector<float> frame;
};

namespace {
constexpr long kCompletedOffset = 20; // after magic, n, steps, every, frames
bool put(std::FILE *f, const void *p, size_t bytes) {
  return std::fwrite(p, 1, bytes, f) == bytes;
}
} // namespace

// Appends a frame already in NBS2 record layout ({x, y, vx, vy} x n, id
// order) and bumps completed_frames.
static int append_frame(nbx_nbs2 *w, const float *rec) {
  if (!put(w->f, rec, 16ull * w->n)) return NBX_ERR_ARG;
  ++w->completed;
  const long end = std::ftell(w->f);
  if (std::fseek(w->f, kCompletedOffset, SEEK_SET) != 0 ||
      !put(w->f, &w->completed, 4) || std::fseek(w->f, end, SEEK_SET) != 0)
    return NBX_ERR_ARG;
  std::fflush(w->f);
  return NBX_OK;
}

extern "C" int nbx_nbs2_open(const char *path, uint32_t n, uint32_t steps,
                             uint32_t every, float dt, const float *mass,
                             const float *radius, nbx_nbs2 **out) {
  if (!path || !out || every == 0 || (n && (!mass || !radius))) return NBX_ERR_ARG;
  *out = nullptr;
  std::FILE *f = std::fopen(path, "wb");
  if (!f) return NBX_ERR_ARG;
  const uint32_t frames = 1 + steps / every, zero = 0;
  const char magic[4] = {'N', 'B', 'S', '2'};
  bool ok = put(f, magic, 4) && put(f, &n, 4) && put(f, &steps, 4) &&
            put(f, &every, 4) && put(f, &frames, 4) && put(f, &zero, 4) &&
            put(f, &dt, 4) && put(f, mass, 4ull * n) && put(f, radius, 4ull * n);
  if (!ok) {
    std::fclose(f);
    return NBX_ERR_ARG;
  }
  nbx_nbs2 *w = new nbx_nbs2();
  w->f = f;
  w->n = n;
  w->frame.resize(4ull * n);
  *out = w;
  return NBX_OK;
}

extern "C" int nbx_nbs2_write_frame(nbx_nbs2 *w, const nbx_body *b) {
  if (!w || (w->n && !b)) return NBX_ERR_ARG;
  for (uint32_t i = 0; i < w->n; ++i) {
    w->frame[4 * i + 0] = b[i].pos_x;
    w->frame[4 * i + 1] = b[i].pos_y;
    w->frame[4 * i + 2] = b[i].vel_x;
    w->frame[4 * i + 3] = b[i].vel_y;
  }
  return append_frame(w, w->frame.data());
}

extern "C" int nbx_nbs2_write_packed(nbx_nbs2 *w, const float *xyvv, uint32_t n) {
  if (!w || n != w->n || (n && !xyvv)) return NBX_ERR_ARG;
  return append_frame(w, xyvv);
}

extern "C" int nbx_nbs2_close(nbx_nbs2 *w) {
  if (!w) return NBX_ERR_ARG;
  const bool ok = std::fclose(w->f) == 0;
  delete w;
  return ok ? NBX_OK : NBX_ERR_ARG;
}
