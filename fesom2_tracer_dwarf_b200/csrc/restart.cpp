// Binary restarts in the reference's derived-type format (restart.hpp).
#include "restart.hpp"

#include <sys/stat.h>
#include <sys/types.h>

#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <stdexcept>

namespace fesom {

namespace {

constexpr int64_t kMaxSubrecord = 2147483639;  // gfortran, 4-byte markers

// ---------------------------------------------------------------------------
// one logical record, built in memory and framed on output
// ---------------------------------------------------------------------------
class RecordOut {
 public:
  void i4(int32_t v) { put(&v, 4); }
  void r8(double v) { put(&v, 8); }
  void l4(bool v) { i4(v ? 1 : 0); }  // default logical: 4 bytes, .true. = 1
  void chars(const std::string &s, size_t len) {
    std::string t = s.substr(0, len);
    t.resize(len, ' ');
    put(t.data(), len);
  }
  // allocatable arrays: extents, then the elements (column-major)
  void arr_i(const std::vector<int32_t> &a, std::initializer_list<int> ext) {
    for (int e : ext) i4(a.empty() ? 0 : e);
    if (!a.empty()) put(a.data(), a.size() * 4);
  }
  void arr_r(const std::vector<double> &a, std::initializer_list<int> ext) {
    for (int e : ext) i4(a.empty() ? 0 : e);
    if (!a.empty()) put(a.data(), a.size() * 8);
  }
  void none(int rank) {  // an unallocated array of the given rank
    for (int q = 0; q < rank; q++) i4(0);
  }
  void static_i(const std::vector<int32_t> &a) {  // write1d_int_static
    i4((int32_t)a.size());
    put(a.data(), a.size() * 4);
  }
  void save(const std::string &path) const {
    std::FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot create " + path + ": " + std::strerror(errno));
    const int64_t n = (int64_t)buf_.size();
    int64_t pos = 0;
    bool first = true;
    do {
      const int64_t len = std::min<int64_t>(kMaxSubrecord, n - pos);
      const bool last = pos + len >= n;
      const int32_t lead = (int32_t)(last ? len : -len), tail = (int32_t)(first ? len : -len);
      bool ok = std::fwrite(&lead, 4, 1, f) == 1;
      ok = ok && (len == 0 || std::fwrite(buf_.data() + pos, 1, (size_t)len, f) == (size_t)len);
      ok = ok && std::fwrite(&tail, 4, 1, f) == 1;
      if (!ok) {
        std::fclose(f);
        throw std::runtime_error("write failed: " + path);
      }
      pos += len;
      first = false;
    } while (pos < n);
    if (std::fclose(f) != 0) throw std::runtime_error("write failed: " + path);
  }

 private:
  void put(const void *p, size_t n) {
    const char *c = static_cast<const char *>(p);
    buf_.insert(buf_.end(), c, c + n);
  }
  std::vector<char> buf_;
};

class RecordIn {
 public:
  explicit RecordIn(const std::string &path) : path_(path) {
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + path + ": " + std::strerror(errno));
    bool more = true;
    while (more) {
      int32_t lead = 0, tail = 0;
      if (std::fread(&lead, 4, 1, f) != 1) fail_file(f, "missing record marker");
      const int64_t len = lead < 0 ? -(int64_t)lead : lead;
      more = lead < 0;
      const size_t at = buf_.size();
      buf_.resize(at + (size_t)len);
      if (len && std::fread(buf_.data() + at, 1, (size_t)len, f) != (size_t)len) fail_file(f, "truncated record");
      if (std::fread(&tail, 4, 1, f) != 1 || (tail < 0 ? -(int64_t)tail : tail) != len)
        fail_file(f, "record markers disagree");
    }
    std::fclose(f);
  }
  int32_t i4(const char *what) { int32_t v; get(&v, 4, what); return v; }
  double r8(const char *what) { double v; get(&v, 8, what); return v; }
  bool l4(const char *what) { return i4(what) != 0; }
  std::string chars(size_t len, const char *what) {
    std::string s(len, ' ');
    get(&s[0], len, what);
    while (!s.empty() && (s.back() == ' ' || s.back() == '\0')) s.pop_back();
    return s;
  }
  // allocatable array of `rank` extents; returns the extents (all zero when
  // unallocated) and fills out
  template <typename T>
  std::vector<int> arr(int rank, std::vector<T> &out, const char *what) {
    std::vector<int> ext(rank);
    size_t n = 1;
    for (int q = 0; q < rank; q++) {
      ext[q] = i4(what);
      if (ext[q] < 0) throw std::runtime_error(path_ + ": negative extent of " + what);
      n *= (size_t)ext[q];
    }
    out.resize(n);
    if (n) get(out.data(), n * sizeof(T), what);
    return ext;
  }
  void skip_arr(int rank, size_t elem, const char *what) {
    size_t n = 1;
    for (int q = 0; q < rank; q++) n *= (size_t)i4(what);
    skip(n * elem, what);
  }
  std::vector<int32_t> static_i(const char *what) {
    const int32_t n = i4(what);
    std::vector<int32_t> v(n > 0 ? n : 0);
    if (n > 0) get(v.data(), 4 * (size_t)n, what);
    return v;
  }
  void skip(size_t n, const char *what) {
    if (pos_ + n > buf_.size()) throw std::runtime_error(path_ + ": record ends inside " + what);
    pos_ += n;
  }
  bool done() const { return pos_ == buf_.size(); }
  const std::string &path() const { return path_; }

 private:
  [[noreturn]] void fail_file(std::FILE *f, const char *why) {
    std::fclose(f);
    throw std::runtime_error(path_ + ": " + why);
  }
  void get(void *p, size_t n, const char *what) {
    if (pos_ + n > buf_.size()) throw std::runtime_error(path_ + ": record ends inside " + what);
    std::memcpy(p, buf_.data() + pos_, n);
    pos_ += n;
  }
  std::string path_;
  std::vector<char> buf_;
  size_t pos_ = 0;
};

void make_dir(const std::string &d) {
  if (mkdir(d.c_str(), 0777) != 0 && errno != EEXIST)
    throw std::runtime_error("cannot create directory " + d + ": " + std::strerror(errno));
}

std::vector<int32_t> one_based(const std::vector<int> &a, bool none_is_zero) {
  std::vector<int32_t> o(a.size());
  for (size_t i = 0; i < a.size(); i++) o[i] = (none_is_zero && a[i] < 0) ? 0 : a[i] + 1;
  return o;
}

const char *kHor[] = {"UPW1", "MUSCL", "MFCT"};
const char *kVer[] = {"UPW1", "PPM", "QR4C", "CDIFF"};
const char *kLim[] = {"NONE", "FCT"};

int scheme_code(const std::string &s, const char *const *names, int n, const char *what) {
  for (int i = 0; i < n; i++)
    if (s == names[i]) return i;
  throw std::runtime_error(std::string("restart: unknown ") + what + " scheme '" + s + "'");
}

// lib/MOD_MESH.F90:185-279
void write_mesh(const std::string &path, const MeshHost &m) {
  const int N = m.nod2D, T = m.elem2D, E = m.edge2D, nl = m.nl, L = nl - 1;
  RecordOut r;
  double ocean_area = 0.0;
  for (int n = 0; n < N; n++) ocean_area += m.area[(size_t)n * nl];
  int edge_in = 0;
  for (int e = 0; e < E; e++) edge_in += m.edge_tri[2 * e + 1] >= 0;
  r.i4(N);
  r.r8(ocean_area);
  r.r8(ocean_area);
  r.i4(E);
  r.i4(edge_in);
  r.i4(T);
  r.arr_i(one_based(m.elem_nodes, false), {3, T});
  r.arr_i(one_based(m.edge_nodes, false), {2, E});
  r.arr_i(one_based(m.edge_tri, true), {2, E});
  r.none(2);  // elem_edges
  r.arr_r(m.elem_area, {T});
  r.arr_r(m.edge_dxdy, {2, E});
  r.arr_r(m.edge_cross, {4, E});
  r.arr_r(m.elem_cos, {T});
  r.none(1);  // metric_factor
  r.none(2);  // elem_neighbors
  // nod_in_elem2D (max_ring, nod2D), zero-padded, and nod_in_elem2D_num
  int maxr = 1;
  for (int n = 0; n < N; n++) maxr = std::max(maxr, m.ring_ptr[n + 1] - m.ring_ptr[n]);
  std::vector<int32_t> nie((size_t)maxr * N, 0), nien(N);
  for (int n = 0; n < N; n++) {
    nien[n] = m.ring_ptr[n + 1] - m.ring_ptr[n];
    for (int p = m.ring_ptr[n]; p < m.ring_ptr[n + 1]; p++) nie[(size_t)n * maxr + (p - m.ring_ptr[n])] = m.ring_elem[p] + 1;
  }
  r.arr_i(nie, {maxr, N});
  r.none(2);  // x_corners
  r.none(2);  // y_corners
  r.arr_i(nien, {N});
  r.none(1);  // depth
  r.none(2);  // gradient_vec
  r.arr_r(m.grad_sca, {6, T});
  r.none(1);  // bc_index_nod2D
  r.i4(nl);
  r.arr_r(m.zbar, {nl});
  r.arr_r(m.Z, {L});
  r.none(1);  // elem_depth
  r.arr_i(std::vector<int32_t>(T, 1), {T});  // ulevels
  r.arr_i(std::vector<int32_t>(N, 1), {N});  // ulevels_nod2D
  r.arr_i(std::vector<int32_t>(N, 1), {N});  // ulevels_nod2D_max
  r.arr_i(std::vector<int32_t>(m.nlev_elem.begin(), m.nlev_elem.end()), {T});
  r.arr_i(std::vector<int32_t>(m.nlev_node.begin(), m.nlev_node.end()), {N});
  r.arr_i(std::vector<int32_t>(m.nlev_node_min.begin(), m.nlev_node_min.end()), {N});
  r.arr_r(m.area, {nl, N});
  r.none(2);  // area_inv
  r.arr_r(m.areasvol, {nl, N});
  r.none(2);  // areasvol_inv
  r.none(1);  // mesh_resolution
  r.none(1);  // cavity_flag_n
  r.none(1);  // cavity_flag_e
  r.none(1);  // cavity_depth
  r.none(2);  // cavity_nrst_cavlpnt_xyz
  r.i4(0);    // ssh_stiff%dim
  r.i4(0);    // ssh_stiff%nza
  for (int q = 0; q < 5; q++) r.none(1);  // rowptr, colind, values, colind_loc, rowptr_loc
  for (int q = 0; q < 4; q++) r.none(1);  // lump2d_south/north, ind_south/north
  r.i4(0);    // nn_size
  r.none(1);  // nn_num
  r.none(2);  // nn_pos
  r.arr_r(m.hnode, {L, N});
  r.arr_r(m.hnode_new, {L, N});
  // zbar_3d_n (nl, nod2D), Z_3d_n (nl-1, nod2D) of the uniform thicknesses
  std::vector<double> zb((size_t)nl * N), zz((size_t)L * N);
  for (int n = 0; n < N; n++) {
    for (int k = 0; k < nl; k++) zb[(size_t)n * nl + k] = m.zbar[k];
    for (int k = 0; k < L; k++) zz[(size_t)n * L + k] = m.Z[k];
  }
  r.arr_r(zb, {nl, N});
  r.arr_r(zz, {L, N});
  r.none(2);  // Z_3d_n_ib
  r.arr_r(m.helem, {L, T});
  for (int q = 0; q < 5; q++) r.none(1);  // bottom_elem/node_thickness, dhe, hbar, hbar_old
  for (int q = 0; q < 4; q++) r.none(1);  // zbar_n_bot, zbar_e_bot, zbar_n_srf, zbar_e_srf
  r.none(1);  // coriolis
  r.none(1);  // coriolis_node
  r.save(path);
}

MeshHost read_mesh(const std::string &path) {
  RecordIn r(path);
  MeshHost m;
  m.nod2D = r.i4("nod2D");
  r.r8("ocean_area");
  r.r8("ocean_areawithcav");
  m.edge2D = r.i4("edge2D");
  r.i4("edge2D_in");
  m.elem2D = r.i4("elem2D");
  const int N = m.nod2D, T = m.elem2D, E = m.edge2D;
  std::vector<int32_t> iv;
  std::vector<double> rv;
  auto need = [&](const std::vector<int> &ext, std::initializer_list<int> want, const char *what) {
    size_t q = 0;
    for (int w : want) {
      if (q >= ext.size() || ext[q] != w)
        throw std::runtime_error(path + ": " + what + " has unexpected extents");
      q++;
    }
  };
  need(r.arr(2, iv, "elem2D_nodes"), {3, T}, "elem2D_nodes");
  m.elem_nodes.assign(iv.begin(), iv.end());
  for (int &x : m.elem_nodes) x -= 1;
  need(r.arr(2, iv, "edges"), {2, E}, "edges");
  m.edge_nodes.assign(iv.begin(), iv.end());
  for (int &x : m.edge_nodes) x -= 1;
  need(r.arr(2, iv, "edge_tri"), {2, E}, "edge_tri");
  m.edge_tri.assign(iv.begin(), iv.end());
  for (int &x : m.edge_tri) x = x > 0 ? x - 1 : -1;
  r.skip_arr(2, 4, "elem_edges");
  need(r.arr(1, m.elem_area, "elem_area"), {T}, "elem_area");
  need(r.arr(2, m.edge_dxdy, "edge_dxdy"), {2, E}, "edge_dxdy");
  need(r.arr(2, m.edge_cross, "edge_cross_dxdy"), {4, E}, "edge_cross_dxdy");
  need(r.arr(1, m.elem_cos, "elem_cos"), {T}, "elem_cos");
  r.skip_arr(1, 8, "metric_factor");
  r.skip_arr(2, 4, "elem_neighbors");
  std::vector<int32_t> nie, nien;
  const std::vector<int> ext_nie = r.arr(2, nie, "nod_in_elem2D");
  r.skip_arr(2, 8, "x_corners");
  r.skip_arr(2, 8, "y_corners");
  need(r.arr(1, nien, "nod_in_elem2D_num"), {N}, "nod_in_elem2D_num");
  if (ext_nie.size() != 2 || ext_nie[1] < N) throw std::runtime_error(path + ": nod_in_elem2D has unexpected extents");
  const int maxr = ext_nie[0];
  m.ring_ptr.assign(N + 1, 0);
  for (int n = 0; n < N; n++) {
    if (nien[n] < 0 || nien[n] > maxr) throw std::runtime_error(path + ": nod_in_elem2D_num out of range");
    m.ring_ptr[n + 1] = m.ring_ptr[n] + nien[n];
  }
  m.ring_elem.resize(m.ring_ptr[N]);
  for (int n = 0; n < N; n++)
    for (int j = 0; j < nien[n]; j++) m.ring_elem[m.ring_ptr[n] + j] = nie[(size_t)n * maxr + j] - 1;
  r.skip_arr(1, 8, "depth");
  r.skip_arr(2, 8, "gradient_vec");
  need(r.arr(2, m.grad_sca, "gradient_sca"), {6, T}, "gradient_sca");
  r.skip_arr(1, 4, "bc_index_nod2D");
  m.nl = r.i4("nl");
  const int nl = m.nl, L = nl - 1;
  if (nl < 3) throw std::runtime_error(path + ": nl < 3");
  need(r.arr(1, m.zbar, "zbar"), {nl}, "zbar");
  need(r.arr(1, m.Z, "Z"), {L}, "Z");
  r.skip_arr(1, 8, "elem_depth");
  for (const char *what : {"ulevels", "ulevels_nod2D", "ulevels_nod2D_max"}) {
    r.arr(1, iv, what);
    for (int32_t u : iv)
      if (u != 1) throw std::runtime_error(path + ": " + what + " /= 1 (cavities) is not supported");
  }
  need(r.arr(1, iv, "nlevels"), {T}, "nlevels");
  m.nlev_elem.assign(iv.begin(), iv.end());
  need(r.arr(1, iv, "nlevels_nod2D"), {N}, "nlevels_nod2D");
  m.nlev_node.assign(iv.begin(), iv.end());
  r.skip_arr(1, 4, "nlevels_nod2D_min");  // recomputed from the rings
  need(r.arr(2, m.area, "area"), {nl, N}, "area");
  r.skip_arr(2, 8, "area_inv");
  need(r.arr(2, m.areasvol, "areasvol"), {nl, N}, "areasvol");
  r.skip_arr(2, 8, "areasvol_inv");
  r.skip_arr(1, 8, "mesh_resolution");
  r.skip_arr(1, 4, "cavity_flag_n");
  r.skip_arr(1, 4, "cavity_flag_e");
  r.skip_arr(1, 8, "cavity_depth");
  r.skip_arr(2, 8, "cavity_nrst_cavlpnt_xyz");
  r.i4("ssh_stiff%dim");
  r.i4("ssh_stiff%nza");
  r.skip_arr(1, 4, "ssh_stiff%rowptr");
  r.skip_arr(1, 4, "ssh_stiff%colind");
  r.skip_arr(1, 8, "ssh_stiff%values");
  r.skip_arr(1, 4, "ssh_stiff%colind_loc");
  r.skip_arr(1, 4, "ssh_stiff%rowptr_loc");
  r.skip_arr(1, 8, "lump2d_south");
  r.skip_arr(1, 8, "lump2d_north");
  r.skip_arr(1, 4, "ind_south");
  r.skip_arr(1, 4, "ind_north");
  r.i4("nn_size");
  r.skip_arr(1, 4, "nn_num");
  r.skip_arr(2, 4, "nn_pos");
  need(r.arr(2, m.hnode, "hnode"), {L, N}, "hnode");
  need(r.arr(2, m.hnode_new, "hnode_new"), {L, N}, "hnode_new");
  r.skip_arr(2, 8, "zbar_3d_n");
  r.skip_arr(2, 8, "Z_3d_n");
  r.skip_arr(2, 8, "Z_3d_n_ib");
  need(r.arr(2, m.helem, "helem"), {L, T}, "helem");
  for (const char *what : {"bottom_elem_thickness", "bottom_node_thickness", "dhe", "hbar", "hbar_old", "zbar_n_bot",
                           "zbar_e_bot", "zbar_n_srf", "zbar_e_srf", "coriolis", "coriolis_node"})
    r.skip_arr(1, 8, what);
  if (!r.done()) throw std::runtime_error(path + ": bytes left after the last field of t_mesh");
  m.coord.assign(2 * (size_t)N, 0.0);  // not part of the record
  return m;
}

// lib/MOD_PARTIT.F90 WRITE_T_COM_STRUCT / WRITE_T_PARTIT (one process)
void write_partit(const std::string &path, const MeshHost &m) {
  RecordOut r;
  for (int c = 0; c < 3; c++) {  // com_nod2D, com_elem2D, com_elem2D_full: no neighbours
    r.i4(0);
    r.static_i(std::vector<int32_t>(32, 0));
    r.static_i(std::vector<int32_t>(33, 0));
    r.none(1);
    r.i4(0);
    r.static_i(std::vector<int32_t>(32, 0));
    r.static_i(std::vector<int32_t>(32, 0));
    r.none(1);
    r.i4(0);
  }
  r.i4(1);    // npes
  r.i4(0);    // mype
  r.i4(100);  // maxPEnum
  r.arr_i(std::vector<int32_t>{1, m.nod2D + 1}, {2});  // part: node ranges per PE
  auto seq = [](int n) {
    std::vector<int32_t> v(n);
    for (int i = 0; i < n; i++) v[i] = i + 1;
    return v;
  };
  r.i4(m.nod2D);
  r.i4(0);
  r.arr_i(seq(m.nod2D), {m.nod2D});
  r.i4(m.elem2D);
  r.i4(0);
  r.i4(0);
  r.arr_i(seq(m.elem2D), {m.elem2D});
  r.i4(m.edge2D);
  r.i4(0);
  r.arr_i(seq(m.edge2D), {m.edge2D});
  r.i4(0);  // pe_status
  r.save(path);
}

void read_partit(const std::string &path, const MeshHost &m) {
  RecordIn r(path);
  std::vector<int32_t> iv;
  for (int c = 0; c < 3; c++) {
    r.i4("rPEnum");
    r.static_i("rPE");
    r.static_i("rptr");
    r.skip_arr(1, 4, "rlist");
    r.i4("sPEnum");
    r.static_i("sPE");
    r.static_i("sptr");
    r.skip_arr(1, 4, "slist");
    r.i4("nreq");
  }
  const int npes = r.i4("npes");
  r.i4("mype");
  r.i4("maxPEnum");
  r.skip_arr(1, 4, "part");
  const int myDim = r.i4("myDim_nod2D"), eDim = r.i4("eDim_nod2D");
  if (npes != 1 || myDim != m.nod2D || eDim != 0)
    throw std::runtime_error(path + ": a partition of " + std::to_string(npes) +
                             " processes; this library reads one-process restarts");
  r.skip_arr(1, 4, "myList_nod2D");
  r.i4("myDim_elem2D");
  r.i4("eDim_elem2D");
  r.i4("eXDim_elem2D");
  r.skip_arr(1, 4, "myList_elem2D");
  r.i4("myDim_edge2D");
  r.i4("eDim_edge2D");
  r.skip_arr(1, 4, "myList_edge2D");
  r.i4("pe_status");
  if (!r.done()) throw std::runtime_error(path + ": bytes left after the last field of t_partit");
}

// lib/MOD_TRACER.F90:104-206
void write_tracers(const std::string &path, const RestartData &d) {
  const MeshHost &m = d.mesh;
  const int N = m.nod2D, E = m.edge2D, L = m.nl - 1;
  RecordOut r;
  const int ntr = (int)d.values.size();
  r.i4(ntr);
  for (int t = 0; t < ntr; t++) {
    r.arr_r(d.values[t], {L, N});
    r.none(3);  // valuesold
    r.arr_r(d.values_ab[t], {L, N});
    r.l4(false);  // smooth_bh_tra
    r.r8(0.0);    // gamma0_tra
    r.r8(0.0);    // gamma1_tra
    r.r8(0.0);    // gamma2_tra
    r.l4(false);  // i_vert_diff
    const TracerScheme &s = d.schemes[t];
    r.chars(kHor[s.hor], 20);
    r.chars(kVer[s.ver], 20);
    r.chars(kLim[s.lim], 20);
    r.r8(s.ph);
    r.r8(s.pv);
    r.i4(d.ids.empty() ? t + 1 : d.ids[t]);
  }
  // work: the 13 step arrays unallocated, then nboundary_lay and edge_up_dn_tri
  for (int q = 0; q < 3; q++) r.none(2);  // del_ttf, del_ttf_advhoriz, del_ttf_advvert
  for (int q = 0; q < 2; q++) r.none(3);  // dvd_trflx_hor, dvd_trflx_ver
  for (int q = 0; q < 7; q++) r.none(2);  // fct_LO .. fct_minus
  r.none(3);                              // edge_up_dn_grad
  r.arr_i(std::vector<int32_t>(m.nboundary_lay.begin(), m.nboundary_lay.end()), {N});
  r.arr_i(one_based(m.up_dn_tri, true), {2, E});
  r.save(path);
}

void read_tracers(const std::string &path, RestartData &d) {
  MeshHost &m = d.mesh;
  const int N = m.nod2D, E = m.edge2D, L = m.nl - 1;
  RecordIn r(path);
  const int ntr = r.i4("num_tracers");
  if (ntr < 0 || ntr > 100000) throw std::runtime_error(path + ": num_tracers out of range");
  for (int t = 0; t < ntr; t++) {
    std::vector<double> v, ab;
    const std::vector<int> ev = r.arr(2, v, "values");
    if (ev[0] != L || ev[1] != N) throw std::runtime_error(path + ": values has unexpected extents");
    r.skip_arr(3, 8, "valuesold");
    const std::vector<int> ea = r.arr(2, ab, "valuesAB");
    if (!ab.empty() && (ea[0] != L || ea[1] != N)) throw std::runtime_error(path + ": valuesAB has unexpected extents");
    if (ab.empty()) ab = v;
    r.l4("smooth_bh_tra");
    r.r8("gamma0_tra");
    r.r8("gamma1_tra");
    r.r8("gamma2_tra");
    r.l4("i_vert_diff");
    TracerScheme s;
    s.hor = scheme_code(r.chars(20, "tra_adv_hor"), kHor, 3, "horizontal");
    s.ver = scheme_code(r.chars(20, "tra_adv_ver"), kVer, 4, "vertical");
    s.lim = scheme_code(r.chars(20, "tra_adv_lim"), kLim, 2, "limiter");
    s.ph = r.r8("tra_adv_ph");
    s.pv = r.r8("tra_adv_pv");
    d.ids.push_back(r.i4("ID"));
    d.values.push_back(std::move(v));
    d.values_ab.push_back(std::move(ab));
    d.schemes.push_back(s);
  }
  for (const char *what : {"del_ttf", "del_ttf_advhoriz", "del_ttf_advvert"}) r.skip_arr(2, 8, what);
  for (const char *what : {"dvd_trflx_hor", "dvd_trflx_ver"}) r.skip_arr(3, 8, what);
  for (const char *what : {"fct_LO", "adv_flux_hor", "adv_flux_ver", "fct_ttf_max", "fct_ttf_min", "fct_plus",
                           "fct_minus"})
    r.skip_arr(2, 8, what);
  r.skip_arr(3, 8, "edge_up_dn_grad");
  std::vector<int32_t> iv;
  const std::vector<int> en = r.arr(1, iv, "nboundary_lay");
  const bool have_nbl = !iv.empty();
  if (have_nbl) {
    if (en[0] != N) throw std::runtime_error(path + ": nboundary_lay has unexpected extents");
    m.nboundary_lay.assign(iv.begin(), iv.end());
  }
  const std::vector<int> eu = r.arr(2, iv, "edge_up_dn_tri");
  const bool have_ud = !iv.empty();
  if (have_ud) {
    if (eu[0] != 2 || eu[1] != E) throw std::runtime_error(path + ": edge_up_dn_tri has unexpected extents");
    m.up_dn_tri.assign(iv.begin(), iv.end());
    for (int &x : m.up_dn_tri) x = x > 0 ? x - 1 : -1;
  }
  if (!r.done()) throw std::runtime_error(path + ": bytes left after the last field of t_tracer");
  if (!have_nbl || !have_ud)
    throw std::runtime_error(path + ": the MUSCL tables (nboundary_lay, edge_up_dn_tri) are not allocated");
}

// lib/MOD_DYN.F90:256-312 (Fer_GM off, as the dwarf never reads the namelist that sets it)
void write_dynamics(const std::string &path, const RestartData &d) {
  const MeshHost &m = d.mesh;
  const int N = m.nod2D, T = m.elem2D, nl = m.nl, L = nl - 1;
  RecordOut r;
  r.i4(5);        // opt_visc
  r.r8(0.03);     // visc_gamma0
  r.r8(0.1);      // visc_gamma1
  r.r8(0.285);    // visc_gamma2
  r.r8(1.5);      // visc_easybsreturn
  r.l4(true);     // use_ivertvisc
  r.i4(2);        // momadv_opt
  r.l4(false);    // use_freeslip
  r.l4(false);    // use_wsplit
  r.r8(1.0);      // wsplit_maxcfl
  r.l4(false);    // use_ssh_se_subcycl
  // solverinfo
  r.i4(1); r.i4(2000); r.i4(15); r.i4(3); r.i4(2);
  r.r8(1.e-8); r.r8(1e-5);
  for (int q = 0; q < 4; q++) r.none(1);
  // work: uvnode_rhs (3D), u_c, v_c, u_b, v_b (2D)
  r.none(3);
  for (int q = 0; q < 4; q++) r.none(2);
  r.arr_r(d.uv, {2, L, T});
  r.none(3);  // uv_rhs
  r.none(4);  // uv_rhsAB
  r.none(3);  // uvnode
  r.arr_r(d.w, {nl, N});
  r.arr_r(d.w, {nl, N});  // w_e
  r.none(2);              // w_i (the step uses w for w_e and w_i alike)
  r.none(2);              // cfl_z
  r.save(path);
}

void read_dynamics(const std::string &path, RestartData &d) {
  const MeshHost &m = d.mesh;
  const int N = m.nod2D, T = m.elem2D, nl = m.nl, L = nl - 1;
  RecordIn r(path);
  r.i4("opt_visc");
  for (const char *what : {"visc_gamma0", "visc_gamma1", "visc_gamma2", "visc_easybsreturn"}) r.r8(what);
  r.l4("use_ivertvisc");
  r.i4("momadv_opt");
  r.l4("use_freeslip");
  r.l4("use_wsplit");
  r.r8("wsplit_maxcfl");
  const bool se = r.l4("use_ssh_se_subcycl");
  for (const char *what : {"ident", "maxiter", "restart", "fillin", "lutype"}) r.i4(what);
  r.r8("droptol");
  r.r8("soltol");
  for (const char *what : {"rr", "zz", "pp", "App"}) r.skip_arr(1, 8, what);
  r.skip_arr(3, 8, "uvnode_rhs");
  for (const char *what : {"u_c", "v_c", "u_b", "v_b"}) r.skip_arr(2, 8, what);
  std::vector<double> uv, w;
  const std::vector<int> eu = r.arr(3, uv, "uv");
  if (!uv.empty() && (eu[0] != 2 || eu[1] != L || eu[2] != T))
    throw std::runtime_error(path + ": uv has unexpected extents");
  r.skip_arr(3, 8, "uv_rhs");
  r.skip_arr(4, 8, "uv_rhsAB");
  r.skip_arr(3, 8, "uvnode");
  const std::vector<int> ew = r.arr(2, w, "w");
  if (!w.empty() && (ew[0] != nl || ew[1] != N)) throw std::runtime_error(path + ": w has unexpected extents");
  for (const char *what : {"w_e", "w_i", "cfl_z"}) r.skip_arr(2, 8, what);
  if (se) {
    r.skip_arr(3, 8, "se_uvh");
    for (const char *what : {"se_uvBT_rhs", "se_uvBT_4AB", "se_uvBT", "se_uvBT_theta", "se_uvBT_mean", "se_uvBT_12",
                             "se_uvBT_stab_hvisc"})
      r.skip_arr(2, 8, what);
    r.skip_arr(1, 8, "se_uvBT_stab_bdrag");
  }
  if (!r.done()) throw std::runtime_error(path + ": bytes left after the last field of t_dynamics");
  if (!uv.empty()) {
    d.uv = std::move(uv);
    d.w = w.empty() ? std::vector<double>((size_t)nl * N, 0.0) : std::move(w);
  }
}

}  // namespace

void write_restart(const std::string &dir, const RestartData &d) {
  make_dir(dir);
  const std::string np = dir + "/np1";
  make_dir(np);
  {
    // lib/io_restart_derivedtype.F90:52-58 (ctarr = 0, 0, 0 as tracer_finalize passes it)
    std::ofstream f(dir + "/meta.time");
    f << "0\n0\n! year: 0\n!   t_mesh\n!   t_partit\n!   t_tracer\n!   t_dynamics\n";
    if (!f) throw std::runtime_error("cannot write " + dir + "/meta.time");
  }
  write_mesh(np + "/t_mesh.0", d.mesh);
  write_partit(np + "/t_partit.0", d.mesh);
  write_tracers(np + "/t_tracer.0", d);
  write_dynamics(np + "/t_dynamics.0", d);
}

RestartData read_restart(const std::string &dir, bool want_tracers, bool want_dynamics) {
  const std::string np = dir + "/np1";
  struct stat st;
  if (stat(np.c_str(), &st) != 0 || !S_ISDIR(st.st_mode))
    throw std::runtime_error("could not find restart directory: " + np);
  RestartData d;
  d.mesh = read_mesh(np + "/t_mesh.0");
  read_partit(np + "/t_partit.0", d.mesh);
  // the MUSCL tables live in the tracer record's work part: read them even
  // when the tracers themselves are not wanted
  const std::string tpath = np + "/t_tracer.0";
  const bool have_tracers = stat(tpath.c_str(), &st) == 0;
  if (want_tracers || have_tracers) read_tracers(tpath, d);
  if (!want_tracers) {
    d.values.clear(); d.values_ab.clear(); d.schemes.clear(); d.ids.clear();
  }
  if (want_dynamics) read_dynamics(np + "/t_dynamics.0", d);
  MeshHost &m = d.mesh;
  m.finalize_tables(false);
  if (m.nboundary_lay.empty()) m.build_nboundary_lay();
  // without a tracer record there are no up/down triangles (the mesh record
  // holds no coordinates to find them): MUSCL then takes the ring means
  if (m.up_dn_tri.empty()) m.up_dn_tri.assign(2 * (size_t)m.edge2D, -1);
  const std::string bad = m.validate();
  if (!bad.empty()) throw std::runtime_error(np + "/t_mesh.0: " + bad);
  return d;
}

}  // namespace fesom
