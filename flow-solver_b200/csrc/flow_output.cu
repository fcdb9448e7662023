// flow_output.cu - result payloads of a solve: the surface pressure
// coefficient files of write_surface_cp (grid_io.C:841-1375) and the Tecplot
// solution files of write_tecplot_solutionC / write_tecplot_solutionP
// (grid_io.C:102-331).
//
// The arithmetic runs on the device over the resident state: the surface
// files need only the wall nodes' pressure coefficients (one small gather
// kernel, a few KB back to the host instead of Q), the Tecplot files one
// packed copy of the real nodes' four values.  The text is formatted on the
// host, split over threads in node order, with the reference's printf
// formats, so the files are byte-identical to the reference's for the same
// state.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "flow_gpu.h"
#include "flow_internal.h"

namespace {

using flow::internal::set_last_error;

// write_surface_cp's pressure coefficient of node nodes[i] from GRID::Q in
// conserved form (grid_io.C:1308-1347): P = (g-1)(e - r(u^2+v^2)/2),
// Cp = (P/p_inf - 1) * 2/(g M^2) with p_inf = 1/g.  Built with --fmad=false,
// the operations round as the reference's.
__global__ void k_surface_cp(const double* __restrict__ Q, const int* __restrict__ nodes,
                             int count, double gamma, double mach, double* __restrict__ cp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const long n = nodes[i];
  const double4 q = reinterpret_cast<const double4*>(Q)[n];
  const double r = q.x;
  const double u = q.y / r;
  const double v = q.z / r;
  const double e = q.w;
  const double P = (gamma - 1.) * (e - 0.5 * r * (u * u + v * v));
  const double pinf = 1. / gamma;
  cp[i] = (P / pinf - 1.) * (2. / (gamma * mach * mach));
}

// Per real node 1..nn the four values a Tecplot file prints: GRID::Q as is
// (conserved, grid_io.C:138-141) or rho, u, v, P (grid_io.C:252-258 for a
// triangle-only mesh, grid_io.C:285-290 otherwise; the two pressure forms
// are the reference's own and differ).
__global__ void k_tecplot_values(const double* __restrict__ Q, int nn, int primitive,
                                 int tri_only, double gamma, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  const double4 q = reinterpret_cast<const double4*>(Q)[i + 1];
  double4 o = q;
  if (primitive) {
    const double rho = q.x;
    const double u = q.y / rho;
    const double v = q.z / rho;
    const double E = q.w;
    double P;
    if (tri_only)
      P = (gamma - 1.) * E - ((gamma - 1.) / 2.) * rho * (u * u + v * v);
    else
      P = (gamma - 1.) * E - ((gamma - 1.) / (2. * rho)) * (u * u + v * v);
    o = make_double4(rho, u, v, P);
  }
  reinterpret_cast<double4*>(out)[i] = o;
}

int cuda_fail(const char* what, cudaError_t e) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  set_last_error(m.c_str());
  return FLOW_ERR_CUDA;
}

// Unique nodes of boundary b's segments in first-appearance order, n0 before
// n1 of each segment (grid_io.C:1294-1349).  seg holds every boundary's
// segments in order, 2 ints each; nbs[b] counts boundary b's.
int boundary_nodes(int nb, const int* nbs, const int* seg, int b, int nn,
                   std::vector<char>& seen, std::vector<int>& out) {
  long first = 0;
  for (int k = 1; k <= nb; k++)
    if (nbs[k] < 0) {
      set_last_error("surface Cp: a boundary has a negative segment count");
      return FLOW_ERR_ARG;
    }
  for (int k = 1; k < b; k++) first += nbs[k];
  for (int s = 0; s < nbs[b]; s++)
    for (int h = 0; h < 2; h++) {
      const int n = seg[2 * (first + s) + h];
      if (n < 1 || n > nn) {
        set_last_error("surface Cp: a boundary segment names a node outside 1..nn");
        return FLOW_ERR_ARG;
      }
      if (!seen[n]) {
        seen[n] = 1;
        out.push_back(n);
      }
    }
  return 0;
}

// Cp of the listed nodes, computed on the context's device and stream (a
// stream-ordered temporary of 12 bytes a node holds the list and the result).
int device_cp(flow_ctx* c, const flow_params* p, const std::vector<int>& nodes,
              std::vector<double>& cp) {
  const double* Q = nullptr;
  int nn = 0, ng = 0;
  if (flow::internal::state_of(c, &Q, &nn, &ng)) {
    set_last_error("surface Cp: null or failed context");
    return FLOW_ERR_ARG;
  }
  cp.assign(nodes.size(), 0.);
  if (nodes.empty()) return 0;
  cudaSetDevice(flow::internal::device_of(c));
  cudaStream_t st = flow::internal::stream_of(c);
  const size_t cnt = nodes.size();
  void* buf = nullptr;
  cudaError_t e = cudaMallocAsync(&buf, cnt * (sizeof(double) + sizeof(int)), st);
  if (e != cudaSuccess) return cuda_fail("surface Cp", e);
  double* d_cp = static_cast<double*>(buf);
  int* d_nodes = reinterpret_cast<int*>(d_cp + cnt);
  e = cudaMemcpyAsync(d_nodes, nodes.data(), cnt * sizeof(int), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    k_surface_cp<<<(unsigned)((cnt + 127) / 128), 128, 0, st>>>(Q, d_nodes, (int)cnt, p->gamma,
                                                               p->mach, d_cp);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(cp.data(), d_cp, cnt * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(buf, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? 0 : cuda_fail("surface Cp", e);
}

// Ordering of `sort -g` under the C locale, which the reference runs over
// each surface file (grid_io.C:1361-1371): by the leading number of the
// line (strtold; a line without one first, NaN before every number), ties
// by the bytes of the whole line.
struct Line {
  long double key;
  int kind;  // 0 no number, 1 NaN, 2 number
  std::string text;
};

bool line_less(const Line& a, const Line& b) {
  if (a.kind != b.kind) return a.kind < b.kind;
  if (a.kind == 2 && a.key != b.key) return a.key < b.key;
  return a.text < b.text;
}

Line make_line(const char* s) {
  Line l;
  l.text = s;
  char* end = nullptr;
  l.key = strtold(l.text.c_str(), &end);
  l.kind = end == l.text.c_str() ? 0 : (std::isnan(l.key) ? 1 : 2);
  return l;
}

// Format nodes [lo, hi) of a Tecplot zone into out.
void format_nodes(const double* x, const double* vals, int lo, int hi, std::string* out) {
  char buf[192];
  out->reserve((size_t)(hi - lo) * 132);
  for (int i = lo; i < hi; i++) {
    const int n = i + 1;
    const double* q = vals + 4 * (size_t)i;
    const int k = snprintf(buf, sizeof(buf), "%.15e %.15e %.15e %.15e %.15e %.15e\n",
                           x[2 * (size_t)n], x[2 * (size_t)n + 1], q[0], q[1], q[2], q[3]);
    out->append(buf, k);
  }
}

}  // namespace

extern "C" {

int flow_surface_cp(flow_ctx* c, const flow_params* p, int nb, const int* nbs, const int* seg,
                    int b, int* nodes_out, double* cp_out, int cap, int* count) {
  if (!c || !p || !nbs || !seg || !count || nb < 1 || b < 1 || b > nb || cap < 0) {
    set_last_error("flow_surface_cp: bad argument");
    return FLOW_ERR_ARG;
  }
  const double* Q = nullptr;
  int nn = 0, ng = 0;
  if (flow::internal::state_of(c, &Q, &nn, &ng)) {
    set_last_error("flow_surface_cp: null or failed context");
    return FLOW_ERR_ARG;
  }
  std::vector<char> seen((size_t)nn + 1, 0);
  std::vector<int> nodes;
  int rc = boundary_nodes(nb, nbs, seg, b, nn, seen, nodes);
  if (rc) return rc;
  *count = (int)nodes.size();
  if ((int)nodes.size() > cap || (!nodes.empty() && (!nodes_out || !cp_out))) {
    set_last_error("flow_surface_cp: output arrays hold fewer entries than the boundary's nodes");
    return FLOW_ERR_ARG;
  }
  std::vector<double> cp;
  rc = device_cp(c, p, nodes, cp);
  if (rc) return rc;
  std::copy(nodes.begin(), nodes.end(), nodes_out);
  std::copy(cp.begin(), cp.end(), cp_out);
  return 0;
}

int flow_write_surface_cp(flow_ctx* c, const flow_params* p, const char* dir, int nb,
                          const int* bbc, const int* nbs, const int* seg, const double* x) {
  if (!c || !p || !bbc || !nbs || !seg || !x || nb < 1) {
    set_last_error("flow_write_surface_cp: bad argument");
    return FLOW_ERR_ARG;
  }
  const double* Q = nullptr;
  int nn = 0, ng = 0;
  if (flow::internal::state_of(c, &Q, &nn, &ng)) {
    set_last_error("flow_write_surface_cp: null or failed context");
    return FLOW_ERR_ARG;
  }
  // every inviscid boundary's nodes (bbc odd, grid_io.C:887) in one device pass
  std::vector<int> nodes, first(nb + 2, 0);
  for (int b = 1; b <= nb; b++) {
    first[b] = (int)nodes.size();
    if (bbc[b] == 0 || bbc[b] % 2 == 0) continue;
    std::vector<char> seen((size_t)nn + 1, 0);
    int rc = boundary_nodes(nb, nbs, seg, b, nn, seen, nodes);
    if (rc) return rc;
  }
  first[nb + 1] = (int)nodes.size();
  std::vector<double> cp;
  int rc = device_cp(c, p, nodes, cp);
  if (rc) return rc;
  const std::string base = (dir && *dir) ? std::string(dir) + "/" : std::string();
  for (int b = 1; b <= nb; b++) {
    if (bbc[b] == 0 || bbc[b] % 2 == 0) continue;
    std::vector<Line> lines;
    lines.reserve(first[b + 1] - first[b]);
    char buf[128];
    for (int i = first[b]; i < first[b + 1]; i++) {
      snprintf(buf, sizeof(buf), "%f  %f\n", (float)x[2 * (size_t)nodes[i]], (float)cp[i]);
      lines.push_back(make_line(buf));
    }
    std::sort(lines.begin(), lines.end(), line_less);
    char name[64];
    snprintf(name, sizeof(name), "surface_%d_pressure.dat", b);
    const std::string path = base + name;
    FILE* fp = fopen(path.c_str(), "w");
    if (!fp) {
      set_last_error(("flow_write_surface_cp: cannot open " + path).c_str());
      return FLOW_ERR_ARG;
    }
    for (const Line& l : lines) fwrite(l.text.data(), 1, l.text.size(), fp);
    if (fclose(fp) != 0) {
      set_last_error(("flow_write_surface_cp: cannot write " + path).c_str());
      return FLOW_ERR_ARG;
    }
  }
  return 0;
}

int flow_write_tecplot(flow_ctx* c, const flow_params* p, const char* path, int primitive,
                       const double* x, int ntri, const int* tri, int nquad, const int* quad) {
  if (!c || !p || !path || !x || ntri < 0 || nquad < 0 || (ntri > 0 && !tri) ||
      (nquad > 0 && !quad)) {
    set_last_error("flow_write_tecplot: bad argument");
    return FLOW_ERR_ARG;
  }
  const double* Q = nullptr;
  int nn = 0, ng = 0;
  if (flow::internal::state_of(c, &Q, &nn, &ng)) {
    set_last_error("flow_write_tecplot: null or failed context");
    return FLOW_ERR_ARG;
  }
  // the node values, packed on the device, then one copy back
  std::vector<double> vals((size_t)nn * 4);
  cudaSetDevice(flow::internal::device_of(c));
  cudaStream_t st = flow::internal::stream_of(c);
  void* buf = nullptr;
  cudaError_t e = cudaMallocAsync(&buf, vals.size() * sizeof(double), st);
  if (e != cudaSuccess) return cuda_fail("flow_write_tecplot", e);
  k_tecplot_values<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(
      Q, nn, primitive ? 1 : 0, nquad == 0 ? 1 : 0, p->gamma, static_cast<double*>(buf));
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(vals.data(), buf, vals.size() * sizeof(double), cudaMemcpyDeviceToHost,
                        st);
  cudaFreeAsync(buf, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail("flow_write_tecplot", e);

  FILE* fp = fopen(path, "w");
  if (!fp) {
    set_last_error((std::string("flow_write_tecplot: cannot open ") + path).c_str());
    return FLOW_ERR_ARG;
  }
  fprintf(fp, "TITLE=\"data file\"\n");
  if (primitive)
    fprintf(fp, "VARIABLES=\"X\", \"Y\", \"Rho\", \"U\", \"V\", \"P\"\n");
  else
    fprintf(fp, "VARIABLES=\"X\", \"Y\", \"Rho\", \"Umom\", \"Vmom\", \"E\"\n");
  if (nquad == 0)
    fprintf(fp, "ZONE N=%d, E=%d, DATAPACKING=POINT, ZONETYPE=FETRIANGLE\n", nn, ntri);
  else
    fprintf(fp, "ZONE N=%d, E=%d, DATAPACKING=POINT, ZONETYPE=FEQUADRILATERAL\n", nn,
            ntri + nquad);
  // node lines, formatted in parallel ranges and written in order
  const int nthr = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const int parts = nn < 4096 ? 1 : nthr;
  std::vector<std::string> text(parts);
  std::vector<std::thread> pool;
  for (int t = 0; t < parts; t++) {
    const int lo = (int)((long)nn * t / parts), hi = (int)((long)nn * (t + 1) / parts);
    pool.emplace_back(format_nodes, x, vals.data(), lo, hi, &text[t]);
  }
  for (auto& th : pool) th.join();
  for (const auto& s : text) fwrite(s.data(), 1, s.size(), fp);
  fprintf(fp, "\n");
  if (nquad == 0) {
    for (int i = 1; i <= ntri; i++)
      fprintf(fp, "%d %d %d\n", tri[i * 3], tri[i * 3 + 1], tri[i * 3 + 2]);
  } else {
    // triangles as degenerate quadrilaterals (last node twice), then the quads
    for (int i = 1; i <= ntri; i++)
      fprintf(fp, "%d %d %d %d\n", tri[i * 3], tri[i * 3 + 1], tri[i * 3 + 2], tri[i * 3 + 2]);
    for (int i = 1; i <= nquad; i++)
      fprintf(fp, "%d %d %d %d\n", quad[i * 4], quad[i * 4 + 1], quad[i * 4 + 2], quad[i * 4 + 3]);
  }
  if (fclose(fp) != 0) {
    set_last_error((std::string("flow_write_tecplot: cannot write ") + path).c_str());
    return FLOW_ERR_ARG;
  }
  return 0;
}

int flow_write_restart(flow_ctx* c, const flow_params* p, const char* path, const double* x,
                       int ntri, const int* tri, int nquad, const int* quad, int nb,
                       const int* nbs, const int* seg) {
  if (!c || !p || !path || !x || ntri < 0 || nquad < 0 || (ntri > 0 && !tri) ||
      (nquad > 0 && !quad) || nb < 1 || !nbs || !seg) {
    set_last_error("flow_write_restart: bad argument");
    return FLOW_ERR_ARG;
  }
  const double* Q = nullptr;
  int nn = 0, ng = 0;
  if (flow::internal::state_of(c, &Q, &nn, &ng)) {
    set_last_error("flow_write_restart: null or failed context");
    return FLOW_ERR_ARG;
  }
  int citer = 0;
  double cfl = 0.;
  int rc = flow::internal::step_position(c, &citer, &cfl);
  if (rc) return rc;
  std::vector<double> q((size_t)(nn + 1) * 4);
  cudaError_t e = cudaMemcpy(q.data(), Q, q.size() * sizeof(double), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail("flow_write_restart", e);
  FILE* fp = fopen(path, "w");
  if (!fp) {
    set_last_error((std::string("flow_write_restart: cannot open ") + path).c_str());
    return FLOW_ERR_ARG;
  }
  // the mesh as write_mesh prints it (mesh_io.C:318-379)
  fprintf(fp, "#Number of grid points\n%d\n", nn);
  for (int n = 1; n <= nn; n++) fprintf(fp, "%.15e %.15e\n", x[2 * n], x[2 * n + 1]);
  fprintf(fp, "#Number of blocks\n%d\n", 1);
  fprintf(fp, "#Number of triangles\n%d\n", ntri);
  for (int i = 1; i <= ntri; i++)
    fprintf(fp, "%d %d %d\n", tri[i * 3], tri[i * 3 + 1], tri[i * 3 + 2]);
  fprintf(fp, "#Number of quads\n%d\n", nquad);
  for (int i = 1; i <= nquad; i++)
    fprintf(fp, "%d %d %d %d\n", quad[i * 4], quad[i * 4 + 1], quad[i * 4 + 2], quad[i * 4 + 3]);
  fprintf(fp, "#Number of boundaries\n%d\n", nb);
  long k = 0;
  for (int b = 1; b <= nb; b++) {
    fprintf(fp, "#Number of edges for boundary %d\n%d\n", b, nbs[b]);
    for (int t = 0; t < nbs[b]; t++, k++) fprintf(fp, "%d %d\n", seg[2 * k], seg[2 * k + 1]);
  }
  // the restart block (mesh_io.C:380-390): step, CFL, the real nodes' Q
  fprintf(fp, "#Number of Constants\n%d\n%d\n%.15E\n", 2, citer, cfl);
  fprintf(fp, "#Number of Variables\n%d\n", 4);
  for (int n = 1; n <= nn; n++)
    fprintf(fp, "%.15e %.15e %.15e %.15e\n", q[4 * (size_t)n], q[4 * (size_t)n + 1],
            q[4 * (size_t)n + 2], q[4 * (size_t)n + 3]);
  if (fclose(fp) != 0) {
    set_last_error((std::string("flow_write_restart: cannot write ") + path).c_str());
    return FLOW_ERR_ARG;
  }
  return 0;
}

}  // extern "C"
