// C++ driver of the ReactorB200 drop-in (pelephysics_b200/csrc/ReactorB200.H),
// in the manner of the reference's ReactEval driver (Testing/Exec/ReactEval/
// main.cpp): one reactor object, created once, reacting host and device data.
//
// Usage: reactor_b200_driver DIR MECH DT
// Reads DIR/in.bin (int32 ncells, N, nx, ny, nz; then doubles rY[ncells][N+1]
// (T in slot N), rX[ncells]; then int32 mask[ncells]) and writes:
//   out_flat.bin     flat react on host arrays, one thread: rY, rX, cost
//   out_threads.bin  the same cells split in two halves reacted concurrently
//                    by two threads on the one object (three rounds): rY, rX
//   out_box.bin      react(Box, Array4...) on device planes with the mask:
//                    rY planes [N][ncells], T, rE, FC
//   out_flatten.bin  flatten of the input box: y_vect [(N+1)][ncells], src_vect,
//                    vect_energy, src_vect_energy
//   out_unflatten.bin unflatten of that y_vect with dt = 0 and FCunt = 7:
//                    rY planes, T, rE, FC
//   out_typ.bin      flat react after set_typ_vals_ode(all 2.0): rY, rX
// and prints print_final_stats of its last call.  Exit status 0 when every
// call returned 0.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "ReactorB200.H"

using ppb_cpp::Array4View;
using ppb_cpp::Box;

static std::vector<char> slurp(const std::string& path)
{
  std::vector<char> b;
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return b;
  std::fseek(f, 0, SEEK_END);
  b.resize((size_t)std::ftell(f));
  std::fseek(f, 0, SEEK_SET);
  if (std::fread(b.data(), 1, b.size(), f) != b.size()) b.clear();
  std::fclose(f);
  return b;
}

static void dump(const std::string& path, const std::vector<std::pair<const void*, size_t>>& parts)
{
  FILE* f = std::fopen(path.c_str(), "wb");
  for (auto& p : parts) std::fwrite(p.first, 1, p.second, f);
  std::fclose(f);
}

#define CK(x)                                                                                                      \
  do {                                                                                                             \
    if ((x) != cudaSuccess) {                                                                                      \
      std::fprintf(stderr, "CUDA error at %s:%d\n", __FILE__, __LINE__);                                         \
      return 2;                                                                                                    \
    }                                                                                                              \
  } while (0)

int main(int argc, char** argv)
{
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s DIR MECH DT\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1];
  const std::string mech = argv[2];
  const double DT = std::atof(argv[3]);
  std::vector<char> in = slurp(dir + "/in.bin");
  if (in.size() < 20) return 2;
  int hdr[5];
  std::memcpy(hdr, in.data(), sizeof(hdr));
  const int nc = hdr[0], N = hdr[1], nx = hdr[2], ny = hdr[3], nz = hdr[4], n = N + 1;
  if (nc != nx * ny * nz) return 2;
  const double* rY0 = (const double*)(in.data() + 20);
  const double* rX0 = rY0 + (size_t)nc * n;
  const int* mask0 = (const int*)(rX0 + nc);

  ppb_cpp::ReactorB200 reactor(mech);
  ppb_options& o = reactor.options();
  o.rtol = 1e-10;
  o.atol = 1e-10;
  o.max_order = 5;
  o.warps_per_block = 8;
  o.team_lanes = 32;
  o.register_budget = 2;
  if (reactor.init(1, nc) != 0) {
    std::fprintf(stderr, "init: %s\n", reactor.last_error());
    return 1;
  }
  int bad = 0;
  std::vector<double> zsrc((size_t)nc * N, 0.0), zx(nc, 0.0);

  // 1. flat react, one thread
  std::vector<double> y(rY0, rY0 + (size_t)nc * n), x(rX0, rX0 + nc);
  double dt = DT, t = 0.0;
  const int cost = reactor.react(y.data(), zsrc.data(), x.data(), zx.data(), dt, t, nc);
  if (cost < 0 || cost == 1) bad++;
  long lcost = cost;
  dump(dir + "/out_flat.bin", {{y.data(), y.size() * 8}, {x.data(), x.size() * 8}, {&lcost, 8}});

  // 2. two threads on the one object, three rounds each
  const int h = nc / 2;
  std::vector<double> ya(rY0, rY0 + (size_t)h * n), xa(rX0, rX0 + h);
  std::vector<double> yb(rY0 + (size_t)h * n, rY0 + (size_t)nc * n), xb(rX0 + h, rX0 + nc);
  int rca = 0, rcb = 0;
  auto worker = [&](std::vector<double>* yy, std::vector<double>* xx, const double* ysrc, const double* xsrc, int m,
                    int* rc) {
    for (int round = 0; round < 3; round++) {
      std::memcpy(yy->data(), ysrc, (size_t)m * n * 8);
      std::memcpy(xx->data(), xsrc, (size_t)m * 8);
      double d = DT, tt = 0.0;
      const int c = reactor.react(yy->data(), zsrc.data(), xx->data(), zx.data(), d, tt, m);
      if (c < 0 || c == 1) *rc = 1;
    }
  };
  std::thread ta(worker, &ya, &xa, rY0, rX0, h, &rca);
  std::thread tb(worker, &yb, &xb, rY0 + (size_t)h * n, rX0 + h, nc - h, &rcb);
  ta.join();
  tb.join();
  bad += rca + rcb;
  dump(dir + "/out_threads.bin",
       {{ya.data(), ya.size() * 8}, {yb.data(), yb.size() * 8}, {xa.data(), xa.size() * 8}, {xb.data(), xb.size() * 8}});

  // 3. the box path on device planes: rY [N][nz][ny][nx], one plane each for
  // T, rE, rEsrc, FC, mask; rYsrc zero
  std::vector<double> hY((size_t)N * nc), hT(nc), hE(nc);
  for (int c = 0; c < nc; c++) {
    for (int k = 0; k < N; k++) hY[(size_t)k * nc + c] = rY0[(size_t)c * n + k];
    hT[c] = rY0[(size_t)c * n + N];
    hE[c] = rX0[c];
  }
  double *dY, *dS, *dT, *dE, *dEs, *dFC;
  int* dM;
  CK(cudaMalloc(&dY, (size_t)N * nc * 8));
  CK(cudaMalloc(&dS, (size_t)N * nc * 8));
  CK(cudaMalloc(&dT, nc * 8));
  CK(cudaMalloc(&dE, nc * 8));
  CK(cudaMalloc(&dEs, nc * 8));
  CK(cudaMalloc(&dFC, nc * 8));
  CK(cudaMalloc(&dM, nc * 4));
  auto upload = [&]() -> int {
    CK(cudaMemcpy(dY, hY.data(), (size_t)N * nc * 8, cudaMemcpyHostToDevice));
    CK(cudaMemset(dS, 0, (size_t)N * nc * 8));
    CK(cudaMemcpy(dT, hT.data(), nc * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dE, hE.data(), nc * 8, cudaMemcpyHostToDevice));
    CK(cudaMemset(dEs, 0, nc * 8));
    CK(cudaMemset(dFC, 0, nc * 8));
    CK(cudaMemcpy(dM, mask0, nc * 4, cudaMemcpyHostToDevice));
    return 0;
  };
  auto plane = [&](double* p, int ncomp) {
    Array4View<double> a;
    a.p = p;
    a.jstride = nx;
    a.kstride = (long)nx * ny;
    a.nstride = nc;
    a.end[0] = nx;
    a.end[1] = ny;
    a.end[2] = nz;
    a.ncomp = ncomp;
    return a;
  };
  auto cplane = [&](double* p, int ncomp) {
    Array4View<const double> a;
    Array4View<double> m = plane(p, ncomp);
    a.p = m.p;
    a.jstride = m.jstride;
    a.kstride = m.kstride;
    a.nstride = m.nstride;
    for (int d = 0; d < 3; d++) a.end[d] = m.end[d];
    a.ncomp = ncomp;
    return a;
  };
  Array4View<int> am;
  am.p = dM;
  am.jstride = nx;
  am.kstride = (long)nx * ny;
  am.nstride = nc;
  am.end[0] = nx;
  am.end[1] = ny;
  am.end[2] = nz;
  const Box box{{0, 0, 0}, {nx - 1, ny - 1, nz - 1}};
  if (upload()) return 2;
  dt = DT;
  t = 0.0;
  if (reactor.react(box, plane(dY, N), plane(dS, N), plane(dT, 1), plane(dE, 1), plane(dEs, 1), plane(dFC, 1), am, dt,
                    t) != 0)
    bad++;
  CK(cudaDeviceSynchronize());
  std::vector<double> oY((size_t)N * nc), oT(nc), oE(nc), oFC(nc);
  CK(cudaMemcpy(oY.data(), dY, oY.size() * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(oT.data(), dT, nc * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(oE.data(), dE, nc * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(oFC.data(), dFC, nc * 8, cudaMemcpyDeviceToHost));
  dump(dir + "/out_box.bin",
       {{oY.data(), oY.size() * 8}, {oT.data(), nc * 8}, {oE.data(), nc * 8}, {oFC.data(), nc * 8}});

  // 4. flatten / unflatten of the input box
  if (upload()) return 2;
  double *yv, *sv, *ev, *esv;
  long* fcu;
  CK(cudaMalloc(&yv, (size_t)n * nc * 8));
  CK(cudaMalloc(&sv, (size_t)N * nc * 8));
  CK(cudaMalloc(&ev, nc * 8));
  CK(cudaMalloc(&esv, nc * 8));
  CK(cudaMalloc(&fcu, nc * 8));
  reactor.flatten(box, nc, cplane(dY, N), cplane(dS, N), cplane(dT, 1), cplane(dE, 1), cplane(dEs, 1), yv, sv, ev, esv);
  if (reactor.last_status() != 0) bad++;
  CK(cudaDeviceSynchronize());
  std::vector<double> fy((size_t)n * nc), fs((size_t)N * nc), fe(nc), fes(nc);
  CK(cudaMemcpy(fy.data(), yv, fy.size() * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(fs.data(), sv, fs.size() * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(fe.data(), ev, nc * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(fes.data(), esv, nc * 8, cudaMemcpyDeviceToHost));
  dump(dir + "/out_flatten.bin",
       {{fy.data(), fy.size() * 8}, {fs.data(), fs.size() * 8}, {fe.data(), nc * 8}, {fes.data(), nc * 8}});
  std::vector<long> seven(nc, 7);
  CK(cudaMemcpy(fcu, seven.data(), nc * 8, cudaMemcpyHostToDevice));
  reactor.unflatten(box, nc, plane(dY, N), plane(dT, 1), plane(dE, 1), plane(dEs, 1), plane(dFC, 1), yv, ev, fcu, 0.0);
  if (reactor.last_status() != 0) bad++;
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(oY.data(), dY, oY.size() * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(oT.data(), dT, nc * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(oE.data(), dE, nc * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(oFC.data(), dFC, nc * 8, cudaMemcpyDeviceToHost));
  dump(dir + "/out_unflatten.bin",
       {{oY.data(), oY.size() * 8}, {oT.data(), nc * 8}, {oE.data(), nc * 8}, {oFC.data(), nc * 8}});

  // 5. typical values, then the flat react again
  if (reactor.set_typ_vals_ode(std::vector<double>(n, 2.0)) != 0) bad++;
  std::vector<double> y2(rY0, rY0 + (size_t)nc * n), x2(rX0, rX0 + nc);
  dt = DT;
  t = 0.0;
  const int c2 = reactor.react(y2.data(), zsrc.data(), x2.data(), zx.data(), dt, t, nc);
  if (c2 < 0 || c2 == 1) bad++;
  dump(dir + "/out_typ.bin", {{y2.data(), y2.size() * 8}, {x2.data(), x2.size() * 8}});
  reactor.print_final_stats(nullptr);
  reactor.close();
  for (void* p : {(void*)dY, (void*)dS, (void*)dT, (void*)dE, (void*)dEs, (void*)dFC, (void*)dM, (void*)yv, (void*)sv,
                  (void*)ev, (void*)esv, (void*)fcu})
    cudaFree(p);
  if (bad) std::fprintf(stderr, "%d call(s) failed: %s\n", bad, reactor.last_error());
  return bad ? 1 : 0;
}
