// nbody_shim.cpp -- the reference's Simulation / QuadTree / collide /
// uniformDisc interfaces implemented over the C ABI (include/nbx.h).
// Every failure of the GPU path throws std::runtime_error with the
// library's message (the reference would exit(1) from CUDA_CHECK).
#include "nbody/Collision.h"
#include "nbody/QuadTree.h"
#include "nbody/Simulation.h"
#include "nbody/Utils.h"
#include "nbx.h"

#include <cstring>
#include <stdexcept>
#include <string>
#include <unordered_map>

struct NbxContext {
  nbx_handle *h = nullptr;
  std::size_t n = 0;
  std::unordered_map<std::uint64_t, Vec2> accByPos; // QuadTree cache

  ~NbxContext() {
    if (h) nbx_destroy(h);
  }
  void check(int rc, const char *what) const {
    if (rc != NBX_OK)
      throw std::runtime_error(std::string(what) + ": " +
                               (h ? nbx_last_error(h) : "nbx error " + std::to_string(rc)));
  }
  // handle for n bodies with the given parameters
  void ensure(std::size_t count, const nbx_params &p) {
    if (!h || n != count) {
      if (h) nbx_destroy(h);
      h = nullptr;
      const uint32_t sz = static_cast<uint32_t>(count);
      check(nbx_create(&p, 1, &sz, &h), "nbx_create");
      n = count;
    } else {
      check(nbx_set_params(h, &p), "nbx_set_params");
    }
  }
  void upload(const std::vector<Body> &b) {
    check(nbx_upload_bodies(h, reinterpret_cast<const nbx_body *>(b.data()), b.size()),
          "nbx_upload_bodies");
  }
  void download(std::vector<Body> &b) {
    check(nbx_download_bodies(h, reinterpret_cast<nbx_body *>(b.data()), b.size(), 0),
          "nbx_download_bodies");
  }
};

namespace {
nbx_params params_for(float dt, float theta, float eps, std::size_t leaf) {
  nbx_params p;
  nbx_params_default(&p);
  p.dt = dt;
  p.theta = theta;
  p.epsilon = eps;
  p.leaf_capacity = static_cast<int32_t>(leaf);
  return p;
}
std::uint64_t pos_key(const Vec2 &v) {
  std::uint32_t a, b;
  std::memcpy(&a, &v.x, 4);
  std::memcpy(&b, &v.y, 4);
  return (std::uint64_t(a) << 32) | b;
}
} // namespace

// ---------------------------------------------------------------- utils
std::vector<Body> uniformDisc(std::size_t n, unsigned seed) {
  std::vector<Body> out(n, Body(Vec2(), Vec2(), 0.0f, 0.0f));
  const int rc = nbx_uniform_disc(static_cast<uint32_t>(n), seed,
                                  reinterpret_cast<nbx_body *>(out.data()));
  if (rc != NBX_OK) throw std::runtime_error("nbx_uniform_disc failed");
  return out;
}

// ------------------------------------------------------------- quadtree
QuadTree::QuadTree(float theta, float epsilon, std::size_t leafCapacity)
    : theta_(theta), epsilon_(epsilon), leaf_(leafCapacity),
      ctx_(new NbxContext()) {}
QuadTree::QuadTree(const QuadTree &o)
    : theta_(o.theta_), epsilon_(o.epsilon_), leaf_(o.leaf_), ctx_(new NbxContext()) {}
QuadTree &QuadTree::operator=(const QuadTree &o) {
  theta_ = o.theta_;
  epsilon_ = o.epsilon_;
  leaf_ = o.leaf_;
  ctx_.reset(new NbxContext());
  return *this;
}
QuadTree::~QuadTree() = default;

void QuadTree::build(std::vector<Body> &bodies) {
  NbxContext &c = *ctx_;
  c.accByPos.clear();
  if (bodies.empty()) return;
  c.ensure(bodies.size(), params_for(0.05f, theta_, epsilon_, leaf_));
  c.upload(bodies);
  c.check(nbx_phase(c.h, NBX_PHASE_ATTRACT), "tree build");
  c.download(bodies);
  c.accByPos.reserve(bodies.size());
  for (const Body &b : bodies) c.accByPos.emplace(pos_key(b.pos), b.acc);
}

Vec2 QuadTree::acceleration(const Vec2 &pos, const std::vector<Body> &) const {
  NbxContext &c = *ctx_;
  auto it = c.accByPos.find(pos_key(pos));
  if (it != c.accByPos.end()) return it->second;
  if (!c.h) return Vec2();
  float ax = 0.0f, ay = 0.0f;
  c.check(nbx_accel_at(c.h, &pos.x, &pos.y, 1, &ax, &ay), "nbx_accel_at");
  return Vec2(ax, ay);
}

// ------------------------------------------------------------ collision
void collide(std::vector<Body> &bodies) {
  // one handle per thread, like the reference's function-local scratch
  static thread_local NbxContext ctx;
  if (bodies.size() < 2) return;
  ctx.ensure(bodies.size(), params_for(0.05f, 1.0f, 1.0f, 16));
  ctx.upload(bodies);
  ctx.check(nbx_phase(ctx.h, NBX_PHASE_COLLIDE), "collide");
  ctx.download(bodies);
}

// ----------------------------------------------------------- simulation
Simulation::Simulation(std::size_t n)
    : dt(0.05f), frame(0), bodies(uniformDisc(n)),
      quadtree(/*theta=*/1.0f, /*epsilon=*/1.0f, /*leafCapacity=*/16),
      ctx_(new NbxContext()) {}

Simulation::~Simulation() = default;

void Simulation::step() {
  if (!bodies.empty()) {
    ctx_->ensure(bodies.size(), params_for(dt, quadtree.theta(), quadtree.epsilon(),
                                           quadtree.leafCapacity()));
    nbx_body *b = reinterpret_cast<nbx_body *>(bodies.data());
    ctx_->check(nbx_step_io(ctx_->h, b, b, bodies.size()), "nbx_step_io");
  }
  frame += 1;
}

void Simulation::attract() {
  if (bodies.empty()) return;
  ctx_->ensure(bodies.size(), params_for(dt, quadtree.theta(), quadtree.epsilon(),
                                         quadtree.leafCapacity()));
  ctx_->upload(bodies);
  ctx_->check(nbx_phase(ctx_->h, NBX_PHASE_ATTRACT), "attract");
  ctx_->download(bodies);
}

void Simulation::iterate() {
  if (bodies.empty()) return;
  ctx_->ensure(bodies.size(), params_for(dt, quadtree.theta(), quadtree.epsilon(),
                                         quadtree.leafCapacity()));
  ctx_->upload(bodies);
  ctx_->check(nbx_phase(ctx_->h, NBX_PHASE_ITERATE), "iterate");
  ctx_->download(bodies);
}

void Simulation::collide() { ::collide(bodies); }
