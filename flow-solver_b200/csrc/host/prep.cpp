// prep.cpp - host preprocessing of a mesh into the grid arrays of the
// nonlinear iteration (include/flow_prep.h).
//
// Every step follows the reference's set-up routine it names, in the same
// order and with the same floating-point operation order, so the resulting
// arrays are those the reference builds.  Where the reference is quadratic
// (the segment -> element search of Build_Boundary_Edge_Data, the subedge
// search of Fix_Subedge_Data, the array shifts of Add_Layer_to_GNSN) the
// same result is produced with hash lookups / per-node lists.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "flow_prep.h"
#include "curved.h"
#include "svd.h"

namespace {

enum { kTri = 1, kQuad = 2 };
enum { kInterior = 0, kBoundary = 1, kGhost = 2 };

thread_local std::string g_prep_error;

}  // namespace

struct flow_mesh {
  int nn = 0, ng = 0, ne = 0, ns = 0, nbe = 0, nb = 0, ntri = 0, nquad = 0, order = 1;
  std::vector<double> x;              // (nn+ng+1)*2
  std::vector<int> tri, quad;         // (n+1)*nv, 1-based rows
  std::vector<int> nbs;               // nb+1
  std::vector<std::vector<std::array<int, 2>>> bs;  // bs[b][s], b,s 1-based
  std::vector<int> seg_flat;          // bs of every boundary in order, 2 per segment
  bool restart = false;               // the file carried a restart block
  int restart_citer = 0;
  double restart_cfl = 0.;
  std::vector<double> restart_q;      // 4 per node, in the file's node order
  std::vector<int> bbc;
  std::vector<int> nn_map;
  std::vector<int> csn, ncsn, nsn, nnsn, esn, edges;
  std::vector<double> el_cent, xn_subedges, xm_subedges, xg_subedges, xn_bedges, xg_bedges,
      xgn_bedges, cv_area, moments, edge_weight;
  std::vector<int> subedges, bedges, bedge_seg, node_order, node_state;
  std::vector<int> ia, iau, ja;
  std::vector<int> gnsn, gnnsn, gnnsn1;
  std::vector<int> svd_m;
  std::vector<long> svd_off;
  std::vector<double> svd_U, svd_VT, svd_S;
};

namespace {

int nverts(int type) { return type == kTri ? 3 : 4; }
int nelem(const flow_mesh& m) { return m.ntri + m.nquad; }
const int* conn(const flow_mesh& m, int type) { return type == kTri ? m.tri.data() : m.quad.data(); }
int* conn(flow_mesh& m, int type) { return type == kTri ? m.tri.data() : m.quad.data(); }
int count(const flow_mesh& m, int type) { return type == kTri ? m.ntri : m.nquad; }
int global_id(const flow_mesh& m, int local, int type) { return type == kTri ? local : local + m.ntri; }

// mesh_utils.C:285-380 RetrieveElementNodesSurroundingVertex
void element_neighbours(const flow_mesh& m, int gelem, int node, int* list) {
  int type = gelem <= m.ntri ? kTri : kQuad;
  int e = type == kTri ? gelem : gelem - m.ntri;
  int nv = nverts(type);
  const int* c = conn(m, type) + (size_t)e * nv;
  int v = 0;
  for (int i = 0; i < nv; i++)
    if (c[i] == node) { v = i; break; }
  if (type == kTri) {
    static const int other[3][2] = {{1, 2}, {0, 2}, {0, 1}};
    list[0] = c[other[v][0]];
    list[1] = c[other[v][1]];
  } else {
    static const int other[4][2] = {{1, 3}, {0, 2}, {1, 3}, {0, 2}};
    list[0] = c[other[v][0]];
    list[1] = c[other[v][1]];
  }
}

// maps.C:35-155 Cells_Surrounding_Node
void cells_surrounding_node(flow_mesh& m) {
  m.ncsn.assign(m.nn + 2, 0);
  for (int type = kTri; type <= kQuad; type++) {
    int nv = nverts(type);
    const int* c = conn(m, type);
    for (int j = 1; j <= count(m, type); j++)
      for (int k = 0; k < nv; k++) m.ncsn[c[j * nv + k] + 1]++;
  }
  for (int i = 1; i <= m.nn + 1; i++) m.ncsn[i] += m.ncsn[i - 1];
  m.csn.assign(m.ncsn[m.nn + 1], 0);
  std::vector<int> pos(m.ncsn.begin(), m.ncsn.end());
  for (int type = kTri; type <= kQuad; type++) {
    int nv = nverts(type);
    const int* c = conn(m, type);
    for (int j = 1; j <= count(m, type); j++)
      for (int k = 0; k < nv; k++) m.csn[pos[c[j * nv + k]]++] = global_id(m, j, type);
  }
}

// maps.C:174-354 Nodes_Surrounding_Node (neighbours in element-traversal order)
void nodes_surrounding_node(flow_mesh& m) {
  m.nnsn.assign(m.nn + 2, 0);
  m.nsn.clear();
  m.nsn.reserve((size_t)m.nn * 7);
  int list[2];
  for (int i = 1; i <= m.nn; i++) {
    int start = (int)m.nsn.size();
    m.nnsn[i] = start;
    for (int j = m.ncsn[i]; j < m.ncsn[i + 1]; j++) {
      element_neighbours(m, m.csn[j], i, list);
      for (int k = 0; k < 2; k++) {
        bool dup = false;
        if (j != m.ncsn[i])
          for (size_t l = start; l < m.nsn.size(); l++)
            if (m.nsn[l] == list[k]) { dup = true; break; }
        if (!dup) m.nsn.push_back(list[k]);
      }
    }
  }
  m.nnsn[m.nn + 1] = (int)m.nsn.size();
}

// maps.C:375-499 Edges_Surrounding_Node (edges L < R in node order)
void edges_surrounding_node(flow_mesh& m) {
  m.ne = 0;
  m.edges.assign(2, 0);
  m.esn.assign(m.nsn.size(), 0);
  for (int i = 1; i <= m.nn; i++) {
    for (int j = m.nnsn[i]; j < m.nnsn[i + 1]; j++) {
      int r = m.nsn[j];
      if (i > r) continue;
      m.ne++;
      m.edges.push_back(i);
      m.edges.push_back(r);
      m.esn[j] = m.ne;
      int k = m.nnsn[r];
      for (; k < m.nnsn[r + 1]; k++)
        if (m.nsn[k] == i) break;
      m.esn[k] = m.ne;
    }
  }
}

struct NodeDeg {
  int id;
  int degree;
};

int compare_degree(const void* a, const void* b) {
  const NodeDeg* x = (const NodeDeg*)a;
  const NodeDeg* y = (const NodeDeg*)b;
  if (x->degree < y->degree) return 1;
  if (x->degree > y->degree) return -1;
  return 0;
}

// reorder.C:58-303 Cuthill_McKee (forward, seeded at the first node of
// maximum degree, each front sorted by descending degree with qsort)
bool cuthill_mckee(flow_mesh& m) {
  cells_surrounding_node(m);
  nodes_surrounding_node(m);
  const int nn = m.nn;
  m.nn_map.assign(nn + 1, 0);
  std::vector<int> queued(nn + 1, 0), R(nn), S(nn);
  int seed = 1;
  int maxdeg = m.nnsn[2] - m.nnsn[1];
  for (int i = 1; i <= nn; i++) {
    int d = m.nnsn[i + 1] - m.nnsn[i];
    if (d > maxdeg) { maxdeg = d; seed = i; }
  }
  int inode = 1, endR = 0, startS = 0, endS = 0;
  m.nn_map[seed] = inode++;
  queued[seed] = 1;
  std::vector<NodeDeg> rn;
  while (inode <= nn) {
    for (int i = m.nnsn[seed]; i < m.nnsn[seed + 1]; i++) {
      int q = m.nsn[i];
      if (!queued[q]) { R[endR++] = q; queued[q] = 1; }
    }
    rn.resize(endR);
    for (int i = 0; i < endR; i++) rn[i] = {R[i], m.nnsn[R[i] + 1] - m.nnsn[R[i]]};
    if (endR > 0) qsort(rn.data(), endR, sizeof(NodeDeg), compare_degree);
    for (int i = 0; i < endR; i++) {
      m.nn_map[rn[i].id] = inode++;
      S[endS++] = rn[i].id;
    }
    endR = 0;
    if (inode > nn) break;
    if (startS >= endS) return false;  // disconnected mesh
    seed = S[startS++];
  }
  std::vector<double> tx((size_t)(nn + 1) * 2, 0.);
  for (int i = 1; i <= nn; i++) {
    tx[(size_t)m.nn_map[i] * 2] = m.x[(size_t)i * 2];
    tx[(size_t)m.nn_map[i] * 2 + 1] = m.x[(size_t)i * 2 + 1];
  }
  for (int i = 1; i <= nn; i++) {
    m.x[(size_t)i * 2] = tx[(size_t)i * 2];
    m.x[(size_t)i * 2 + 1] = tx[(size_t)i * 2 + 1];
  }
  for (int type = kTri; type <= kQuad; type++) {
    int nv = nverts(type);
    int* c = conn(m, type);
    for (int j = 1; j <= count(m, type); j++)
      for (int k = 0; k < nv; k++) c[j * nv + k] = m.nn_map[c[j * nv + k]];
  }
  for (int b = 1; b <= m.nb; b++)
    for (int s = 1; s <= m.nbs[b]; s++) {
      m.bs[b][s][0] = m.nn_map[m.bs[b][s][0]];
      m.bs[b][s][1] = m.nn_map[m.bs[b][s][1]];
    }
  return true;
}

// geometry.C:31-104 Find_Element_Centroids
void element_centroids(flow_mesh& m) {
  m.el_cent.assign((size_t)(nelem(m) + 1) * 2, 0.);
  for (int type = kTri; type <= kQuad; type++) {
    int nv = nverts(type);
    const int* c = conn(m, type);
    for (int j = 1; j <= count(m, type); j++) {
      double xc = 0., yc = 0.;
      for (int k = 0; k < nv; k++) {
        xc += m.x[2 * c[j * nv + k]];
        yc += m.x[2 * c[j * nv + k] + 1];
      }
      xc /= (nv * 1.);
      yc /= (nv * 1.);
      int g = global_id(m, j, type);
      m.el_cent[2 * g] = xc;
      m.el_cent[2 * g + 1] = yc;
    }
  }
}

// geometry.C:119-391 Build_Edge_Data (one subedge per element side)
bool build_edge_data(flow_mesh& m) {
  int ts = m.ntri * 3 + m.nquad * 4;
  m.subedges.assign((size_t)(ts + 1) * 2, 0);
  m.xn_subedges.assign((size_t)(ts + 1) * 3, 0.);
  m.xm_subedges.assign((size_t)(ts + 1) * 2, 0.);
  std::vector<int> hits(m.ne + 1, 0);
  int is = 0;
  for (int type = kTri; type <= kQuad; type++) {
    int nv = nverts(type);
    const int* c = conn(m, type);
    for (int j = 1; j <= count(m, type); j++) {
      int g = global_id(m, j, type);
      double xc = m.el_cent[2 * g], yc = m.el_cent[2 * g + 1];
      for (int k = 0; k < nv; k++) {
        is++;
        int L = c[j * nv + k], R = c[j * nv + (k + 1) % nv];
        if (L > R) { int t = L; L = R; R = t; }
        double xmid = 0.5 * (m.x[2 * L] + m.x[2 * R]);
        double ymid = 0.5 * (m.x[2 * L + 1] + m.x[2 * R + 1]);
        int iedge = 0;
        for (int n = m.nnsn[L]; n < m.nnsn[L + 1]; n++) {
          iedge = m.esn[n];
          if (m.edges[2 * iedge + 1] == R) break;
        }
        double nx = yc - ymid, ny = xmid - xc;
        if (R == c[j * nv + k]) { nx = -nx; ny = -ny; }
        m.subedges[2 * is] = iedge;
        m.subedges[2 * is + 1] = g;
        m.xn_subedges[3 * is] = nx;
        m.xn_subedges[3 * is + 1] = ny;
        m.xm_subedges[2 * is] = xmid;
        m.xm_subedges[2 * is + 1] = ymid;
        hits[iedge]++;
      }
    }
  }
  m.ns = is;
  for (int i = 1; i <= m.ne; i++)
    if (hits[i] < 1 || hits[i] > 2) return false;
  for (int i = 1; i <= m.ns; i++) {
    double* v = &m.xn_subedges[3 * i];
    double mag = sqrt(v[0] * v[0] + v[1] * v[1]);
    if (mag > 1.0E-20) { v[0] /= mag; v[1] /= mag; }
    v[2] = mag;
  }
  return true;
}

// geometry.C:407-835 Build_Boundary_Edge_Data (two half-segment bedges and
// two ghost nodes per boundary segment)
bool build_boundary_edge_data(flow_mesh& m) {
  int tb = 0;
  for (int b = 1; b <= m.nb; b++) tb += m.nbs[b];
  tb *= 2;
  m.nbe = tb;
  m.ng = tb;
  m.x.resize((size_t)(m.nn + m.ng + 1) * 2, 0.);
  m.node_state.assign(m.nn + m.ng + 1, kInterior);
  m.bedges.assign((size_t)(tb + 1) * 5, 0);
  m.bedge_seg.assign((size_t)(tb + 1) * 2, 0);
  m.xn_bedges.assign((size_t)(tb + 1) * 3, 0.);
  int ib = 1, gh = 1;
  for (int b = 1; b <= m.nb; b++) {
    for (int s = 1; s <= m.nbs[b]; s++) {
      int n0 = m.bs[b][s][0], n1 = m.bs[b][s][1];
      int bc = m.bbc[b];
      m.node_state[n0] = kBoundary;
      m.node_state[n1] = kBoundary;
      double* x = m.x.data();
      if (bc <= 10) {
        double xmid = (x[2 * n0] + x[2 * n1]) / 2.;
        double ymid = (x[2 * n0 + 1] + x[2 * n1 + 1]) / 2.;
        double nx = x[2 * n1 + 1] - ymid;
        double ny = xmid - x[2 * n1];
        for (int h = 0; h < 2; h++) {
          int node = h ? n1 : n0;
          m.bedges[ib * 5] = node;
          m.bedges[ib * 5 + 1] = gh;
          m.bedges[ib * 5 + 3] = b;
          m.bedges[ib * 5 + 4] = s;
          m.xn_bedges[ib * 3] = nx;
          m.xn_bedges[ib * 3 + 1] = ny;
          x[2 * (m.nn + gh)] = (x[2 * node] + xmid) / 2.;
          x[2 * (m.nn + gh) + 1] = (x[2 * node + 1] + ymid) / 2.;
          m.node_state[m.nn + gh] = kGhost;
          ib++;
          gh++;
        }
      } else {
        double xL[2] = {x[2 * n0], x[2 * n0 + 1]}, xR[2] = {x[2 * n1], x[2 * n1 + 1]}, xM[2];
        flow_curved_midpoint(bc, xL, xR, xM);
        for (int h = 0; h < 2; h++) {
          int node = h ? n1 : n0;
          double nx, ny;
          flow_curved_normal(bc, h ? xR : xL, &nx, &ny);
          m.bedges[ib * 5] = node;
          m.bedges[ib * 5 + 1] = gh;
          m.bedges[ib * 5 + 3] = b;
          m.bedges[ib * 5 + 4] = s;
          m.xn_bedges[ib * 3] = nx;
          m.xn_bedges[ib * 3 + 1] = ny;
          x[2 * (m.nn + gh)] = xM[0];
          x[2 * (m.nn + gh) + 1] = xM[1];
          m.node_state[m.nn + gh] = kGhost;
          ib++;
          gh++;
        }
      }
    }
  }
  // element owning each segment: the first element (triangles first) in
  // which n0 -> n1 are consecutive vertices (geometry.C:732-772)
  // Only the segments' keys are looked up: elements are scanned in order
  // (triangles, then quads, each ascending) and a key keeps its first owner;
  // edges that do not start at a boundary node cannot be a segment.
  std::unordered_map<long long, int> owner;  // segment key -> element (0: none yet)
  owner.reserve((size_t)m.nbe * 2);
  for (int i = 1; i <= m.nbe; i++) {
    int b = m.bedges[i * 5 + 3], s = m.bedges[i * 5 + 4];
    owner.emplace((long long)m.bs[b][s][0] * (m.nn + 1) + m.bs[b][s][1], 0);
  }
  for (int type = kTri; type <= kQuad; type++) {
    int nv = nverts(type);
    const int* c = conn(m, type);
    for (int j = 1; j <= count(m, type); j++)
      for (int k = 0; k < nv; k++) {
        const int a = c[j * nv + k];
        if (m.node_state[a] != kBoundary) continue;
        auto it = owner.find((long long)a * (m.nn + 1) + c[j * nv + (k + 1) % nv]);
        if (it != owner.end() && it->second == 0) it->second = global_id(m, j, type);
      }
  }
  for (int i = 1; i <= m.nbe; i++) {
    int b = m.bedges[i * 5 + 3], s = m.bedges[i * 5 + 4];
    int n0 = m.bs[b][s][0], n1 = m.bs[b][s][1];
    auto it = owner.find((long long)n0 * (m.nn + 1) + n1);
    if (it == owner.end() || it->second == 0) return false;
    m.bedges[i * 5 + 2] = it->second;
    m.bedge_seg[i * 2] = n0;
    m.bedge_seg[i * 2 + 1] = n1;
  }
  for (int i = 1; i <= m.nbe; i++) {
    double* v = &m.xn_bedges[3 * i];
    double mag = sqrt(v[0] * v[0] + v[1] * v[1]);
    int bc = m.bbc[m.bedges[i * 5 + 3]];
    if (bc > 10) {
      int node = m.bedges[i * 5], ghost = m.bedges[i * 5 + 1] + m.nn;
      double xL[2] = {m.x[2 * node], m.x[2 * node + 1]};
      double xR[2] = {m.x[2 * ghost], m.x[2 * ghost + 1]};
      flow_curved_arclength(bc, xL, xR, &mag);
      v[2] = mag;
    } else {
      if (mag > 1.0E-20) { v[0] /= mag; v[1] /= mag; }
      v[2] = mag;
    }
  }
  return true;
}

// geometry.C:852-981 Fix_Subedge_Data: the dual face of a subedge on a
// curved segment ends at the curve midpoint, not the chord midpoint.
bool fix_subedge_data(flow_mesh& m) {
  bool any = false;
  for (int b = 1; b <= m.nb; b++)
    if (m.bbc[b] > 10) any = true;
  if (!any) return true;
  // unordered node pair of each curved segment -> its first subedge (lowest
  // index); only edges joining two boundary nodes can be a segment's
  std::unordered_map<long long, int> first_sub;
  auto pair_key = [&](int a, int c) {
    return (long long)std::min(a, c) * (m.nn + 1) + std::max(a, c);
  };
  for (int i = 1; i <= m.nbe; i++) {
    int b = m.bedges[i * 5 + 3], s = m.bedges[i * 5 + 4];
    if (m.bbc[b] > 10) first_sub.emplace(pair_key(m.bs[b][s][0], m.bs[b][s][1]), 0);
  }
  for (int j = 1; j <= m.ns; j++) {
    int e = m.subedges[2 * j];
    int a = m.edges[2 * e], c = m.edges[2 * e + 1];
    if (m.node_state[a] != kBoundary || m.node_state[c] != kBoundary) continue;
    auto it = first_sub.find(pair_key(a, c));
    if (it != first_sub.end() && it->second == 0) it->second = j;
  }
  for (int i = 1; i <= m.nbe; i++) {
    int ghost = m.bedges[i * 5 + 1], gelem = m.bedges[i * 5 + 2];
    int b = m.bedges[i * 5 + 3], s = m.bedges[i * 5 + 4];
    if (m.bbc[b] <= 10) continue;
    int nL = m.bs[b][s][0], nR = m.bs[b][s][1];
    auto it = first_sub.find(pair_key(nL, nR));
    if (it == first_sub.end() || it->second == 0) return false;
    int j = it->second;
    if (m.subedges[2 * j + 1] != gelem) return false;
    double XC0 = m.el_cent[2 * gelem], XC1 = m.el_cent[2 * gelem + 1];
    double XM0 = m.x[2 * (m.nn + ghost)], XM1 = m.x[2 * (m.nn + ghost) + 1];
    double nx = XC1 - XM1, ny = XM0 - XC0;
    double len = sqrt(nx * nx + ny * ny);
    nx /= len;
    ny /= len;
    if (nL > nR) { nx = -nx; ny = -ny; }
    m.xn_subedges[3 * j] = nx;
    m.xn_subedges[3 * j + 1] = ny;
    m.xn_subedges[3 * j + 2] = len;
    m.xm_subedges[2 * j] = XM0;
    m.xm_subedges[2 * j + 1] = XM1;
  }
  return true;
}

// 3-point Gauss points on the segment xL -> xR (geometry.C:1071-1090)
void gauss3(double xL, double yL, double xR, double yR, double* gp) {
  const double t1 = sqrt(15.0) / 5.0, t2 = 0., t3 = sqrt(15.0) / (-5.0);
  gp[0] = (xL + xR) * 0.5 + (xR - xL) * 0.5 * t1;
  gp[1] = (yL + yR) * 0.5 + (yR - yL) * 0.5 * t1;
  gp[2] = (xL + xR) * 0.5 + (xR - xL) * 0.5 * t2;
  gp[3] = (yL + yR) * 0.5 + (yR - yL) * 0.5 * t2;
  gp[4] = (xL + xR) * 0.5 + (xR - xL) * 0.5 * t3;
  gp[5] = (yL + yR) * 0.5 + (yR - yL) * 0.5 * t3;
}

// geometry.C:993-1197 Generate_Gaussian_Data_For_Edge
void gaussian_data(flow_mesh& m) {
  m.xg_subedges.assign((size_t)(m.ns + 1) * 6, 0.);
  m.xg_bedges.assign((size_t)(m.nbe + 1) * 6, 0.);
  m.xgn_bedges.assign((size_t)(m.nbe + 1) * 9, 0.);
  for (int s = 1; s <= m.ns; s++) {
    int g = m.subedges[2 * s + 1];
    gauss3(m.xm_subedges[2 * s], m.xm_subedges[2 * s + 1], m.el_cent[2 * g], m.el_cent[2 * g + 1],
           &m.xg_subedges[6 * s]);
  }
  for (int i = 1; i <= m.nbe; i++) {
    int rn = m.bedges[i * 5], gn = m.bedges[i * 5 + 1] + m.nn;
    double nx = m.xn_bedges[3 * i], ny = m.xn_bedges[3 * i + 1], len = m.xn_bedges[3 * i + 2];
    int b = m.bedges[i * 5 + 3], s = m.bedges[i * 5 + 4];
    int bc = m.bbc[b];
    int nodeL = m.bs[b][s][0], nodeR = m.bs[b][s][1];
    double xi = m.x[2 * rn], yi = m.x[2 * rn + 1];
    double xmid = 0.5 * (m.x[2 * nodeL] + m.x[2 * nodeR]);
    double ymid = 0.5 * (m.x[2 * nodeL + 1] + m.x[2 * nodeR + 1]);
    if (bc <= 10) {
      if (rn == nodeL) gauss3(xi, yi, xmid, ymid, &m.xg_bedges[6 * i]);
      else gauss3(xmid, ymid, xi, yi, &m.xg_bedges[6 * i]);
      for (int k = 0; k < 3; k++) {
        m.xgn_bedges[9 * i + 3 * k] = nx;
        m.xgn_bedges[9 * i + 3 * k + 1] = ny;
        m.xgn_bedges[9 * i + 3 * k + 2] = len;
      }
    } else {
      double XL[2], XR[2], GP[6];
      if (rn == nodeL) {
        XL[0] = m.x[2 * rn]; XL[1] = m.x[2 * rn + 1];
        XR[0] = m.x[2 * gn]; XR[1] = m.x[2 * gn + 1];
      } else {
        XR[0] = m.x[2 * rn]; XR[1] = m.x[2 * rn + 1];
        XL[0] = m.x[2 * gn]; XL[1] = m.x[2 * gn + 1];
      }
      flow_curved_gauss_points(bc, XL, XR, GP);
      flow_curved_arclength(bc, XL, XR, &len);
      for (int j = 0; j < 3; j++) {
        flow_curved_normal(bc, &GP[2 * j], &nx, &ny);
        m.xg_bedges[6 * i + 2 * j] = GP[2 * j];
        m.xg_bedges[6 * i + 2 * j + 1] = GP[2 * j + 1];
        m.xgn_bedges[9 * i + 3 * j] = nx;
        m.xgn_bedges[9 * i + 3 * j + 1] = ny;
        m.xgn_bedges[9 * i + 3 * j + 2] = len;
      }
    }
  }
}

// cv_calc.C:34-232 cv_calc_area_Green (divergence theorem on the median dual)
void cv_area_green(flow_mesh& m) {
  m.cv_area.assign(m.nn + 1, 0.);
  for (int i = 1; i <= m.ns; i++) {
    int e = m.subedges[2 * i], g = m.subedges[2 * i + 1];
    int L = m.edges[2 * e], R = m.edges[2 * e + 1];
    double xc = m.el_cent[2 * g];
    double nx = m.xn_subedges[3 * i], len = m.xn_subedges[3 * i + 2];
    double xmid = m.xm_subedges[2 * i];
    m.cv_area[L] += (xc + xmid) / 2. * nx * len;
    m.cv_area[R] -= (xc + xmid) / 2. * nx * len;
  }
  const double w[3] = {8. / 9., 5. / 9., 5. / 9.};
  for (int b = 1; b <= m.nb; b++) {
    for (int s = 1; s <= m.nbs[b]; s++) {
      int n0 = m.bs[b][s][0], n1 = m.bs[b][s][1];
      int bc = m.bbc[b];
      const double* x = m.x.data();
      if (bc <= 10) {
        double ymid = (x[2 * n0 + 1] + x[2 * n1 + 1]) / 2.;
        double nx = x[2 * n1 + 1] - ymid;
        m.cv_area[n0] += (0.75 * x[2 * n0] + 0.25 * x[2 * n1]) * nx;
        m.cv_area[n1] += (0.75 * x[2 * n1] + 0.25 * x[2 * n0]) * nx;
      } else {
        double xL[2] = {x[2 * n0], x[2 * n0 + 1]}, xR[2] = {x[2 * n1], x[2 * n1 + 1]}, xM[2];
        double GP[6], nx, ny, len;
        flow_curved_midpoint(bc, xL, xR, xM);
        for (int h = 0; h < 2; h++) {
          double F = 0.;
          if (h == 0) flow_curved_gauss_points(bc, xL, xM, GP);
          else flow_curved_gauss_points(bc, xM, xR, GP);
          for (int k = 0; k < 3; k++) {
            flow_curved_normal(bc, &GP[2 * k], &nx, &ny);
            F += (w[k] * GP[2 * k] * nx);
          }
          if (h == 0) flow_curved_arclength(bc, xL, xM, &len);
          else flow_curved_arclength(bc, xM, xR, &len);
          F = F * len * 0.5;
          m.cv_area[h ? n1 : n0] += F;
        }
      }
    }
  }
}

// The nine boundary moment integrals of one straight piece (cv_calc.C:1130-1210)
void moment_terms(double x1, double y1, double x2, double y2, double x3, double y3, double xi,
                  double yi, double nx, double len, double* I) {
  const double w1 = 5. / 9., w2 = 8. / 9., w3 = w1;
  double Ix = w1 * (x1 - xi) * (x1 - xi) + w2 * (x2 - xi) * (x2 - xi) + w3 * (x3 - xi) * (x3 - xi);
  I[0] = 0.5 * Ix * nx * len / 2.;
  double Iy = w1 * (x1 - xi) * (y1 - yi) + w2 * (x2 - xi) * (y2 - yi) + w3 * (x3 - xi) * (y3 - yi);
  I[1] = Iy * nx * len / 2.;
  double Ixx = w1 * (x1 - xi) * (x1 - xi) * (x1 - xi) + w2 * (x2 - xi) * (x2 - xi) * (x2 - xi) +
               w3 * (x3 - xi) * (x3 - xi) * (x3 - xi);
  I[2] = (1. / 3.) * Ixx * nx * len / 2.;
  double Iyy = w1 * (x1 - xi) * (y1 - yi) * (y1 - yi) + w2 * (x2 - xi) * (y2 - yi) * (y2 - yi) +
               w3 * (x3 - xi) * (y3 - yi) * (y3 - yi);
  I[3] = Iyy * nx * len / 2.;
  double Ixy = w1 * (x1 - xi) * (x1 - xi) * (y1 - yi) + w2 * (x2 - xi) * (x2 - xi) * (y2 - yi) +
               w3 * (x3 - xi) * (x3 - xi) * (y3 - yi);
  I[4] = 0.5 * Ixy * nx * len / 2.;
  double Ixxx = w1 * (x1 - xi) * (x1 - xi) * (x1 - xi) * (x1 - xi) +
                w2 * (x2 - xi) * (x2 - xi) * (x2 - xi) * (x2 - xi) +
                w3 * (x3 - xi) * (x3 - xi) * (x3 - xi) * (x3 - xi);
  I[5] = (0.25) * Ixxx * nx * len / 2.;
  double Iyyy = w1 * (x1 - xi) * (y1 - yi) * (y1 - yi) * (y1 - yi) +
                w2 * (x2 - xi) * (y2 - yi) * (y2 - yi) * (y2 - yi) +
                w3 * (x3 - xi) * (y3 - yi) * (y3 - yi) * (y3 - yi);
  I[6] = Iyyy * nx * len / 2.;
  double Ixxy = w1 * (x1 - xi) * (x1 - xi) * (x1 - xi) * (y1 - yi) +
                w2 * (x2 - xi) * (x2 - xi) * (x2 - xi) * (y2 - yi) +
                w3 * (x3 - xi) * (x3 - xi) * (x3 - xi) * (y3 - yi);
  I[7] = (1. / 3.) * Ixxy * nx * len / 2.;
  double Ixyy = w1 * (x1 - xi) * (x1 - xi) * (y1 - yi) * (y1 - yi) +
                w2 * (x2 - xi) * (x2 - xi) * (y2 - yi) * (y2 - yi) +
                w3 * (x3 - xi) * (x3 - xi) * (y3 - yi) * (y3 - yi);
  I[8] = 0.5 * Ixyy * nx * len / 2.;
}

// cv_calc.C:981-1860 cv_calc_Moments: CV moments about the node from the
// divergence theorem, divided by the CV area.  (The area-integral cross
// check that the reference also evaluates only feeds its debug output.)
void cv_moments(flow_mesh& m) {
  m.moments.assign((size_t)(m.nn + 1) * 9, 0.);
  double I[9], gp[6];
  for (int i = 1; i <= m.ns; i++) {
    int e = m.subedges[2 * i], g = m.subedges[2 * i + 1];
    int L = m.edges[2 * e], R = m.edges[2 * e + 1];
    double xc = m.el_cent[2 * g], yc = m.el_cent[2 * g + 1];
    double nx = m.xn_subedges[3 * i], len = m.xn_subedges[3 * i + 2];
    double xmid = m.xm_subedges[2 * i], ymid = m.xm_subedges[2 * i + 1];
    gauss3(xmid, ymid, xc, yc, gp);
    moment_terms(gp[0], gp[1], gp[2], gp[3], gp[4], gp[5], m.x[2 * L], m.x[2 * L + 1], nx, len, I);
    for (int k = 0; k < 9; k++) m.moments[(size_t)L * 9 + k] += I[k];
    moment_terms(gp[0], gp[1], gp[2], gp[3], gp[4], gp[5], m.x[2 * R], m.x[2 * R + 1], nx, len, I);
    for (int k = 0; k < 9; k++) m.moments[(size_t)R * 9 + k] -= I[k];
  }
  const double w[3] = {8. / 9., 5. / 9., 5. / 9.};
  for (int i = 1; i <= m.nbe; i++) {
    int node = m.bedges[i * 5], b = m.bedges[i * 5 + 3], s = m.bedges[i * 5 + 4];
    int bc = m.bbc[b];
    int nodeL = m.bs[b][s][0], nodeR = m.bs[b][s][1];
    double xi = m.x[2 * node], yi = m.x[2 * node + 1];
    if (bc <= 10) {
      double xmid = 0.5 * (m.x[2 * nodeL] + m.x[2 * nodeR]);
      double ymid = 0.5 * (m.x[2 * nodeL + 1] + m.x[2 * nodeR + 1]);
      double len = m.xn_bedges[3 * i + 2], nx = m.xn_bedges[3 * i];
      if (node == nodeL) gauss3(xi, yi, xmid, ymid, gp);
      else gauss3(xmid, ymid, xi, yi, gp);
      moment_terms(gp[0], gp[1], gp[2], gp[3], gp[4], gp[5], xi, yi, nx, len, I);
      for (int k = 0; k < 9; k++) m.moments[(size_t)node * 9 + k] += I[k];
    } else {
      double XL[2] = {m.x[2 * nodeL], m.x[2 * nodeL + 1]}, XR[2] = {m.x[2 * nodeR], m.x[2 * nodeR + 1]};
      double XM[2], GP[6], len, nx, ny;
      flow_curved_midpoint(bc, XL, XR, XM);
      if (node == nodeL) {
        XL[0] = xi; XL[1] = yi; XR[0] = XM[0]; XR[1] = XM[1];
      } else {
        XL[0] = XM[0]; XL[1] = XM[1]; XR[0] = xi; XR[1] = yi;
      }
      flow_curved_gauss_points(bc, XL, XR, GP);
      flow_curved_arclength(bc, XL, XR, &len);
      double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int k = 0; k < 3; k++) {
        flow_curved_normal(bc, &GP[2 * k], &nx, &ny);
        double a = GP[2 * k] - xi, c = GP[2 * k + 1] - yi;
        J[0] += (w[k] * a * a * nx * len);
        J[1] += (w[k] * a * c * nx * len);
        J[2] += (w[k] * a * a * a * nx * len);
        J[3] += (w[k] * a * c * c * nx * len);
        J[4] += (w[k] * a * a * c * nx * len);
        J[5] += (w[k] * a * a * a * a * nx * len);
        J[6] += (w[k] * a * c * c * c * nx * len);
        J[7] += (w[k] * a * a * a * c * nx * len);
        J[8] += (w[k] * a * a * c * c * nx * len);
      }
      I[0] = 0.5 * J[0] * 0.5;
      I[1] = J[1] * 0.5;
      I[2] = (1. / 3.) * J[2] * 0.5;
      I[3] = J[3] * 0.5;
      I[4] = 0.5 * J[4] * 0.5;
      I[5] = (0.25) * J[5] * 0.5;
      I[6] = J[6] * 0.5;
      I[7] = (1. / 3.) * J[7] * 0.5;
      I[8] = 0.5 * J[8] * 0.5;
      for (int k = 0; k < 9; k++) m.moments[(size_t)node * 9 + k] += I[k];
    }
  }
  for (int i = 1; i <= m.nn; i++)
    for (int k = 0; k < 9; k++) m.moments[(size_t)i * 9 + k] /= m.cv_area[i];
}

// init_memory.C:36-138 Build_CRS (row = neighbours in nsn order, then the node)
void build_crs(flow_mesh& m) {
  m.ia.assign(m.nn + 2, 0);
  m.iau.assign(m.nn + 1, 0);
  for (int n = 1; n <= m.nn + 1; n++) m.ia[n] = m.nnsn[n] + (n - 1);
  for (int n = 1; n <= m.nn; n++) m.iau[n] = m.ia[n + 1] - 1;
  m.ja.clear();
  m.ja.reserve(m.nsn.size() + m.nn);
  for (int n = 1; n <= m.nn; n++) {
    for (int j = m.nnsn[n]; j < m.nnsn[n + 1]; j++) m.ja.push_back(m.nsn[j]);
    m.ja.push_back(n);
  }
}

// gradient.C:923-1121 Compute_Edge_Weights (unweighted 2x2 normal equations)
void edge_weights(flow_mesh& m) {
  std::vector<double> r11(m.nn + 1, 0.), r12(m.nn + 1, 0.), s22(m.nn + 1, 0.), r22o(m.nn + 1, 0.);
  for (int i = 1; i <= m.ne; i++) {
    int L = m.edges[2 * i], R = m.edges[2 * i + 1];
    double d0 = m.x[2 * R] - m.x[2 * L], d1 = m.x[2 * R + 1] - m.x[2 * L + 1];
    double t = d0 * d0;
    r11[L] += t;
    r11[R] += t;
    t = d0 * d1;
    r12[L] += t;
    t = (-d0) * (-d1);
    r12[R] += t;
    t = d1 * d1;
    s22[L] += t;
    s22[R] += t;
  }
  for (int i = 1; i <= m.nn; i++) r22o[i] = s22[i] - (r12[i] * r12[i]) / r11[i];
  m.edge_weight.assign((size_t)(m.ne + 1) * 4, 0.);
  for (int i = 1; i <= m.ne; i++) {
    int L = m.edges[2 * i], R = m.edges[2 * i + 1];
    double d0 = m.x[2 * R] - m.x[2 * L], d1 = m.x[2 * R + 1] - m.x[2 * L + 1];
    double* w = &m.edge_weight[4 * i];
    w[1] = (+d1 - r12[L] / r11[L] * (+d0)) / r22o[L];
    w[0] = (+d0 - r12[L] * w[1]) / r11[L];
    w[3] = (-d1 - r12[R] / r11[R] * (-d0)) / r22o[R];
    w[2] = (-d0 - r12[R] * w[3]) / r11[R];
  }
}

// body(lo, hi) over the nodes [1, n], in contiguous ranges on up to 16 host
// threads; for work that is independent per node, so the split does not
// change any result.
template <class F>
void for_node_ranges(int n, F&& body) {
  const int hw = (int)std::thread::hardware_concurrency();
  const int parts = n < 8192 ? 1 : std::max(1, std::min(hw, 16));
  if (parts == 1) {
    body(1, n + 1);
    return;
  }
  std::vector<std::thread> pool;
  for (int t = 0; t < parts; t++) {
    const int lo = 1 + (int)((long)n * t / parts), hi = 1 + (int)((long)n * (t + 1) / parts);
    pool.emplace_back([&body, lo, hi] { body(lo, hi); });
  }
  for (auto& th : pool) th.join();
}

// maps.C:1181-1551 generic layered stencils, grown as solve.C:57-114 does on
// the first third-order step: one layer for every node, a second for every
// node of order > 2, then up to three more for nodes with fewer than six
// neighbours.  Layout identical to the reference's gnsn/gnnsn/gnnsn1.
bool build_stencils(flow_mesh& m) {
  const int nn = m.nn;
  std::vector<std::vector<std::vector<int>>> layers(nn + 1);
  auto add_layer = [&](int i) {
    auto& L = layers[i];
    const auto& last = L.back();
    std::vector<int> cand;
    for (int nb : last)
      for (int j = m.nnsn[nb]; j < m.nnsn[nb + 1]; j++) {
        int e = m.esn[j];
        int a = m.edges[2 * e], b = m.edges[2 * e + 1];
        cand.push_back(a != nb ? a : b);
      }
    std::vector<int> add;
    for (int c : cand) {
      bool f = false;
      for (const auto& lay : L) {
        for (int q : lay)
          if (q == c) { f = true; break; }
        if (f) break;
      }
      if (!f)
        for (int q : add)
          if (q == c) { f = true; break; }
      if (!f) add.push_back(c);
    }
    L.push_back(add);
  };
  auto nnb = [&](int i) {
    int n = 0;
    for (size_t l = 1; l < layers[i].size(); l++) n += (int)layers[i][l].size();
    return n;
  };
  // a node's layers depend only on the mesh and its own earlier layers, so
  // each node runs the three growth passes in turn, nodes in parallel
  std::atomic<bool> ok(true);
  for_node_ranges(nn, [&](int lo, int hi) {
    for (int i = lo; i < hi; i++) {
      layers[i].push_back({i});
      add_layer(i);
      if (m.node_order[i] > 2) add_layer(i);
      if (m.node_order[i] < 3) continue;
      int k = 0;
      for (; nnb(i) < 6 && k < 3; k++) add_layer(i);
      if (nnb(i) < 6) ok = false;
    }
  });
  if (!ok) return false;
  m.gnsn.clear();
  m.gnnsn.assign(1, 0);
  m.gnnsn1.assign(nn + 2, 0);
  for (int i = 1; i <= nn; i++) {
    m.gnnsn1[i] = (int)m.gnnsn.size();
    for (const auto& lay : layers[i]) {
      m.gnnsn.push_back((int)m.gnsn.size());
      for (int q : lay) m.gnsn.push_back(q);
    }
  }
  m.gnnsn1[nn + 1] = (int)m.gnnsn.size();
  m.gnnsn.push_back((int)m.gnsn.size());
  return true;
}

// compute_derivatives.C:848-940: weighted reduced 5-column LSQ matrix of each
// node's stencil (moments shift the monomials to CV averages), factored by SVD.
bool factor_stencils(flow_mesh& m) {
  const int nn = m.nn;
  m.svd_m.assign(nn + 1, 0);
  m.svd_off.assign(nn + 1, 0);
  m.svd_U.clear();
  m.svd_VT.assign((size_t)(nn + 1) * 25, 0.);
  m.svd_S.assign((size_t)(nn + 1) * 5, 0.);
  const double* x = m.x.data();
  const double* mo = m.moments.data();
  // U blocks in node order: offsets first, then each node factored on its own
  long total = 0;
  for (int i = 1; i <= nn; i++) {
    if (m.node_order[i] < 3) continue;
    const int mr = m.gnnsn[m.gnnsn1[i + 1]] - m.gnnsn[m.gnnsn1[i] + 1];
    m.svd_m[i] = mr;
    m.svd_off[i] = total;
    total += 5L * mr;
  }
  m.svd_U.assign((size_t)total, 0.);
  std::atomic<bool> ok(true);
  for_node_ranges(nn, [&](int lo, int hi) {
  std::vector<double> A;
  for (int i = lo; i < hi; i++) {
    if (m.node_order[i] < 3) continue;
    int a0 = m.gnnsn[m.gnnsn1[i] + 1], a1 = m.gnnsn[m.gnnsn1[i + 1]];
    int mr = a1 - a0;
    A.assign((size_t)mr * 5, 0.);
    for (int j = a0; j < a1; j++) {
      int node = m.gnsn[j];
      double dx0 = x[node * 2] - x[i * 2], dx1 = x[node * 2 + 1] - x[i * 2 + 1];
      double dist = sqrt(dx0 * dx0 + dx1 * dx1);
      double w = 1.0 / pow(dist, 1.0);
      int row = j - a0;
      A[row + 0 * mr] = w * (x[node * 2] - x[i * 2] + mo[node * 9 + 0] - mo[i * 9 + 0]);
      A[row + 1 * mr] = w * (x[node * 2 + 1] - x[i * 2 + 1] + mo[node * 9 + 1] - mo[i * 9 + 1]);
      A[row + 2 * mr] = 0.5 * w *
                        ((x[node * 2] - x[i * 2]) * (x[node * 2] - x[i * 2]) +
                         2.0 * mo[node * 9 + 0] * (x[node * 2] - x[i * 2]) + mo[node * 9 + 2] -
                         mo[i * 9 + 2]);
      A[row + 3 * mr] = 0.5 * w *
                        ((x[node * 2 + 1] - x[i * 2 + 1]) * (x[node * 2 + 1] - x[i * 2 + 1]) +
                         2.0 * mo[node * 9 + 1] * (x[node * 2 + 1] - x[i * 2 + 1]) +
                         mo[node * 9 + 3] - mo[i * 9 + 3]);
      A[row + 4 * mr] = w * (mo[node * 9 + 4] + mo[node * 9 + 0] * (x[node * 2 + 1] - x[i * 2 + 1]) +
                             mo[node * 9 + 1] * (x[node * 2] - x[i * 2]) +
                             (x[node * 2 + 1] - x[i * 2 + 1]) * (x[node * 2] - x[i * 2]) -
                             mo[i * 9 + 4]);
    }
    if (flow_svd_jacobi(mr, 5, A.data(), &m.svd_S[(size_t)i * 5], &m.svd_U[m.svd_off[i]],
                        &m.svd_VT[(size_t)i * 25], 0) != 0)
      ok = false;
  }
  });
  return ok;
}

flow_mesh* finish(flow_mesh* m, int reorder, int order, int* status) {
  auto fail = [&](const char* msg) -> flow_mesh* {
    g_prep_error = msg;
    if (status) *status = FLOW_ERR_ARG;
    delete m;
    return nullptr;
  };
  m->order = order;
  if (reorder) {
    if (!cuthill_mckee(*m)) return fail("Cuthill-McKee: the mesh is not connected");
  } else {
    m->nn_map.assign(m->nn + 1, 0);
    for (int i = 0; i <= m->nn; i++) m->nn_map[i] = i;
  }
  cells_surrounding_node(*m);
  nodes_surrounding_node(*m);
  edges_surrounding_node(*m);
  element_centroids(*m);
  if (!build_edge_data(*m)) return fail("an edge borders neither one nor two elements");
  if (!build_boundary_edge_data(*m)) return fail("a boundary segment has no element on its left");
  if (!fix_subedge_data(*m)) return fail("curved segment without its subedge");
  gaussian_data(*m);
  cv_area_green(*m);
  for (int i = 1; i <= m->nn; i++)
    if (!(m->cv_area[i] > 0.)) return fail("non-positive control-volume area");
  cv_moments(*m);
  build_crs(*m);
  m->node_order.assign(m->nn + m->ng + 1, 0);
  for (int i = 1; i <= m->nn; i++) m->node_order[i] = order;
  for (int i = 1; i <= m->nbe; i++)
    m->node_order[m->bedges[i * 5 + 1] + m->nn] = m->node_order[m->bedges[i * 5]];
  edge_weights(*m);  // k=1, and the second-order start-up steps of k=2
  if (order == 3) {
    if (!build_stencils(*m)) return fail("a node's stencil stays below 6 neighbours");
    if (!factor_stencils(*m)) return fail("SVD of a stencil failed");
  }
  m->seg_flat.clear();
  for (int b = 1; b <= m->nb; b++)
    for (int t = 1; t <= m->nbs[b]; t++) {
      m->seg_flat.push_back(m->bs[b][t][0]);
      m->seg_flat.push_back(m->bs[b][t][1]);
    }
  if (status) *status = 0;
  return m;
}

}  // namespace

extern "C" {

flow_mesh* flow_prep_build(int nn, const double* x, int ntri, const int* tri, int nquad,
                           const int* quad, int nb, const int* nbs, const int* seg, const int* bbc,
                           int reorder, int order, int* status) {
  if (nn < 3 || !x || ntri < 0 || nquad < 0 || nb < 1 || !nbs || !seg || !bbc ||
      (order != 1 && order != 3)) {
    g_prep_error = "bad arguments";
    if (status) *status = FLOW_ERR_ARG;
    return nullptr;
  }
  flow_mesh* m = new flow_mesh();
  m->nn = nn;
  m->ntri = ntri;
  m->nquad = nquad;
  m->nb = nb;
  m->x.assign((size_t)(nn + 1) * 2, 0.);
  for (int i = 0; i < nn; i++) {
    m->x[(size_t)(i + 1) * 2] = x[2 * i];
    m->x[(size_t)(i + 1) * 2 + 1] = x[2 * i + 1];
  }
  m->tri.assign((size_t)(ntri + 1) * 3, 0);
  for (int t = 0; t < ntri * 3; t++) m->tri[3 + t] = tri[t];
  m->quad.assign((size_t)(nquad + 1) * 4, 0);
  for (int t = 0; t < nquad * 4; t++) m->quad[4 + t] = quad[t];
  m->nbs.assign(nb + 1, 0);
  m->bbc.assign(nb + 1, 0);
  m->bs.assign(nb + 1, {});
  int k = 0;
  for (int b = 1; b <= nb; b++) {
    m->nbs[b] = nbs[b - 1];
    m->bbc[b] = bbc[b - 1];
    m->bs[b].assign(nbs[b - 1] + 1, {0, 0});
    for (int s = 1; s <= nbs[b - 1]; s++, k++) m->bs[b][s] = {seg[2 * k], seg[2 * k + 1]};
  }
  return finish(m, reorder, order, status);
}

flow_mesh* flow_prep_read(const char* path, const int* bbc, int nb_bc, int reorder, int order,
                          int* status) {
  FILE* fp = fopen(path, "r");
  if (!fp) {
    g_prep_error = "cannot open mesh file";
    if (status) *status = FLOW_ERR_ARG;
    return nullptr;
  }
  char buf[256];
  auto line = [&]() -> bool { return fgets(buf, sizeof(buf), fp) != nullptr; };
  // n numbers from the line, in order (strtod / strtol: the conversions
  // scanf's %lf / %d make, without its per-call format parsing)
  auto doubles = [&](double* out, int n) -> bool {
    char* p = buf;
    for (int k = 0; k < n; k++) {
      char* e = nullptr;
      out[k] = strtod(p, &e);
      if (e == p) return false;
      p = e;
    }
    return true;
  };
  auto ints = [&](int* out, int n) -> bool {
    char* p = buf;
    for (int k = 0; k < n; k++) {
      char* e = nullptr;
      out[k] = (int)strtol(p, &e, 10);
      if (e == p) return false;
      p = e;
    }
    return true;
  };
  auto read_int = [&](int* v) -> bool { return line() && line() && ints(v, 1); };
  int nn = 0, nblk = 0, ntri = 0, nquad = 0, nb = 0;
  bool ok = read_int(&nn) && nn > 0;
  std::vector<double> x;
  std::vector<int> tri, quad, nbs, seg;
  if (ok) {
    x.resize((size_t)nn * 2);
    for (int i = 0; i < nn && ok; i++)
      ok = line() && doubles(&x[2 * i], 2);
  }
  ok = ok && read_int(&nblk) && nblk == 1 && read_int(&ntri) && ntri >= 0;
  if (ok) {
    tri.resize((size_t)ntri * 3);
    for (int t = 0; t < ntri && ok; t++)
      ok = line() && ints(&tri[3 * t], 3);
  }
  ok = ok && read_int(&nquad) && nquad >= 0;
  if (ok) {
    quad.resize((size_t)nquad * 4);
    for (int t = 0; t < nquad && ok; t++)
      ok = line() && ints(&quad[4 * t], 4);
  }
  ok = ok && read_int(&nb) && nb >= 1 && nb == nb_bc;
  for (int b = 0; b < nb && ok; b++) {
    int n = 0;
    ok = read_int(&n) && n >= 1;
    nbs.push_back(n);
    for (int s = 0; s < n && ok; s++) {
      int ac[2] = {0, 0};
      ok = line() && ints(ac, 2);
      seg.push_back(ac[0]);
      seg.push_back(ac[1]);
    }
  }
  // an optional restart block, as write_mesh appends it (mesh_io.C:380-390,
  // read back by mesh_io.C:217-262): constants (the last step, its CFL) and
  // the conserved variables of every node, in the file's node order
  bool restart = false;
  int r_citer = 0;
  double r_cfl = 0.;
  std::vector<double> r_q;
  auto blank = [&]() {
    for (const char* q = buf; *q; q++)
      if (*q != ' ' && *q != '\t' && *q != '\r' && *q != '\n') return false;
    return true;
  };
  bool more = false;  // a comment line after the boundaries opens the block
  while (ok && line()) {
    if (blank()) continue;
    more = buf[0] == '#';
    break;
  }
  if (more) {
    int nconst = 0, nvar = 0;
    bool rok = line() && ints(&nconst, 1) && nconst == 2 && line() && ints(&r_citer, 1) &&
               line() && doubles(&r_cfl, 1) && read_int(&nvar) && nvar == 4;
    if (rok) {
      r_q.resize((size_t)nn * 4);
      for (int i = 0; i < nn && rok; i++) rok = line() && doubles(&r_q[4 * (size_t)i], 4);
    }
    if (!rok) ok = false;
    restart = rok;
  }
  fclose(fp);
  if (!ok) {
    g_prep_error = "malformed mesh file, restart block or boundary count differs from bc list";
    if (status) *status = FLOW_ERR_ARG;
    return nullptr;
  }
  flow_mesh* m = flow_prep_build(nn, x.data(), ntri, tri.data(), nquad, quad.data(), nb,
                                 nbs.data(), seg.data(), bbc, reorder, order, status);
  if (m && restart) {
    m->restart = true;
    m->restart_citer = r_citer;
    m->restart_cfl = r_cfl;
    m->restart_q = std::move(r_q);
  }
  return m;
}

int flow_prep_restart_state(const flow_mesh* m, double* Q, long nQ, int* citer, double* cfl) {
  if (!m || !Q || nQ < (long)(m->nn + m->ng + 1) * 4) return FLOW_ERR_ARG;
  if (!m->restart) {
    g_prep_error = "the mesh file had no restart block";
    return FLOW_ERR_NOT_FOUND;
  }
  std::fill(Q, Q + (size_t)(m->nn + m->ng + 1) * 4, 0.);
  // the file's node i is node nn_map[i] after the renumbering (none when the
  // file is read without reordering, as the reference reads a restart)
  for (int i = 1; i <= m->nn; i++)
    for (int v = 0; v < 4; v++) Q[4 * (size_t)m->nn_map[i] + v] = m->restart_q[4 * (size_t)(i - 1) + v];
  // ghosts copied from their real node (main.C:602-622, ic.C:84-96)
  for (int i = 1; i <= m->nbe; i++) {
    const int n = m->bedges[i * 5], g = m->bedges[i * 5 + 1] + m->nn;
    for (int v = 0; v < 4; v++) Q[4 * (size_t)g + v] = Q[4 * (size_t)n + v];
  }
  if (citer) *citer = m->restart_citer;
  if (cfl) *cfl = m->restart_cfl;
  return 0;
}

int flow_prep_view(const flow_mesh* m, flow_grid_view* v) {
  if (!m || !v) return FLOW_ERR_ARG;
  memset(v, 0, sizeof(*v));
  v->nn = m->nn;
  v->nn_ghost = m->ng;
  v->nedges = m->ne;
  v->nsubedges = m->ns;
  v->nbedges = m->nbe;
  v->nb = m->nb;
  v->nelem = m->ntri + m->nquad;
  v->edges = m->edges.data();
  v->subedges = m->subedges.data();
  v->bedges = m->bedges.data();
  v->bedge_seg = m->bedge_seg.data();
  v->bbc = m->bbc.data();
  v->node_order = m->node_order.data();
  v->ia = m->ia.data();
  v->iau = m->iau.data();
  v->ja = m->ja.data();
  v->x = m->x.data();
  v->cv_area = m->cv_area.data();
  v->el_cent = m->el_cent.data();
  v->xn_subedges = m->xn_subedges.data();
  v->xm_subedges = m->xm_subedges.data();
  v->xg_subedges = m->xg_subedges.data();
  v->xn_bedges = m->xn_bedges.data();
  v->xg_bedges = m->xg_bedges.data();
  v->xgn_bedges = m->xgn_bedges.data();
  v->edge_weight = m->edge_weight.empty() ? nullptr : m->edge_weight.data();
  v->moments = m->moments.data();
  if (m->order == 3) {
    v->gnsn = m->gnsn.data();
    v->gnnsn = m->gnnsn.data();
    v->gnnsn1 = m->gnnsn1.data();
    v->svd_m = m->svd_m.data();
    v->svd_off = m->svd_off.data();
    v->svd_U = m->svd_U.data();
    v->svd_VT = m->svd_VT.data();
    v->svd_S = m->svd_S.data();
  }
  return 0;
}

int flow_prep_initial_state(const flow_mesh* m, const flow_params* p, double* Q) {
  if (!m || !p || !Q) return FLOW_ERR_ARG;
  double angle = p->alpha * M_PI / 180.;
  double rho = 1.0, c = 1.0;
  double P = rho * c * c / p->gamma;
  double u = p->mach * cos(angle), v = p->mach * sin(angle);
  double et = P / (p->gamma - 1.0) + 0.5 * rho * (u * u + v * v);
  size_t tot = (size_t)(m->nn + m->ng + 1) * 4;
  for (size_t i = 0; i < tot; i++) Q[i] = 0.;
  for (int n = 1; n <= m->nn; n++) {
    Q[4 * n] = rho;
    Q[4 * n + 1] = rho * u;
    Q[4 * n + 2] = rho * v;
    Q[4 * n + 3] = et;
  }
  for (int i = 1; i <= m->nbe; i++) {
    int n = m->bedges[i * 5], g = m->bedges[i * 5 + 1] + m->nn;
    for (int k = 0; k < 4; k++) Q[4 * g + k] = Q[4 * n + k];
  }
  return 0;
}

const int* flow_prep_node_map(const flow_mesh* m) { return m ? m->nn_map.data() : nullptr; }

int flow_prep_elements(const flow_mesh* m, int* ntri, const int** tri, int* nquad,
                       const int** quad) {
  if (!m || !ntri || !tri || !nquad || !quad) return FLOW_ERR_ARG;
  *ntri = m->ntri;
  *tri = m->tri.data();
  *nquad = m->nquad;
  *quad = m->quad.data();
  return 0;
}

int flow_prep_segments(const flow_mesh* m, int* nb, const int** bbc, const int** nbs,
                       const int** seg) {
  if (!m || !nb || !bbc || !nbs || !seg) return FLOW_ERR_ARG;
  *nb = m->nb;
  *bbc = m->bbc.data();
  *nbs = m->nbs.data();
  *seg = m->seg_flat.data();
  return 0;
}

void flow_prep_free(flow_mesh* m) { delete m; }

const char* flow_prep_last_error(void) { return g_prep_error.c_str(); }

}  // extern "C"
