// gauge_io.cu -- gauge-field configuration files and the plaquette / link-trace
// measurements their headers carry.
//
// The reference reads its configurations with Grid's NerscIO::readConfiguration
// (src/Test_wilsonclover_mg_lime.cc:75) or IldgReader (:61-68,
// src/Test_wilsonclover_mg.cc:96-99) and writes them with
// NerscIO::writeConfiguration (src/Test_wilson_cg_unprec.cc:72).  Grid is not
// part of the reference; the two formats are restated here from their
// published descriptions:
//
// NERSC archive format: an ASCII header of "KEY = VALUE" lines between
// BEGIN_HEADER and END_HEADER, then the links site by site (x fastest), the
// four directions of a site in order, each link row-major as (re, im) pairs,
// in the byte order and width FLOATING_POINT names (IEEE32BIG, IEEE64BIG,
// IEEE32LITTLE, IEEE64LITTLE).  DATATYPE 4D_SU3_GAUGE_3x3 stores all three
// rows; 4D_SU3_GAUGE stores the first two, the third being the complex
// conjugate of their cross product (an SU(3) matrix's unitarity).  CHECKSUM
// is the sum, modulo 2^32, of the stored payload read as 32-bit words in the
// file's byte order; PLAQUETTE is the average over sites and the six planes
// of Re tr(U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag) / 3 and LINK_TRACE
// the average of Re tr U_mu(x) / 3.
//
// ILDG files are LIME containers: records of a 144-byte big-endian header
// (magic 0x456789ab, version, begin/end flags, 64-bit payload length, a
// 128-byte type string) followed by the payload padded to 8 bytes.  The
// "ildg-format" record is XML naming the precision (32 or 64) and the lattice
// extents lx, ly, lz, lt; the "ildg-binary-data" record holds the 3 x 3 links
// big-endian in the NERSC site and direction order.
//
// The in-memory layout is the library's gauge layout: [site][mu][3][3]
// complex128, sites lexicographic with x fastest.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <sstream>

#include "gmg_internal.cuh"

namespace gmg {
namespace gio {

inline bool host_big_endian() {
  const uint16_t one = 1;
  return *reinterpret_cast<const uint8_t*>(&one) == 0;
}

template <class W> W bswap(W v) {
  uint8_t b[sizeof(W)];
  std::memcpy(b, &v, sizeof(W));
  for (size_t i = 0; i < sizeof(W) / 2; ++i) std::swap(b[i], b[sizeof(W) - 1 - i]);
  std::memcpy(&v, b, sizeof(W));
  return v;
}

// 32-bit word sum of a byte range in the file's byte order
uint32_t word_sum(const unsigned char* p, size_t n, bool big) {
  uint32_t s = 0;
  for (size_t k = 0; k + 4 <= n; k += 4) {
    uint32_t w;
    std::memcpy(&w, p + k, 4);
    if (big != host_big_endian()) w = bswap(w);
    s += w;
  }
  return s;
}

double read_real(const unsigned char* p, int prec, bool big) {
  if (prec == 64) {
    uint64_t u;
    std::memcpy(&u, p, 8);
    if (big != host_big_endian()) u = bswap(u);
    double d;
    std::memcpy(&d, &u, 8);
    return d;
  }
  uint32_t u;
  std::memcpy(&u, p, 4);
  if (big != host_big_endian()) u = bswap(u);
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

void write_real(unsigned char* p, double v, int prec, bool big) {
  if (prec == 64) {
    uint64_t u;
    std::memcpy(&u, &v, 8);
    if (big != host_big_endian()) u = bswap(u);
    std::memcpy(p, &u, 8);
  } else {
    const float f = (float)v;
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if (big != host_big_endian()) u = bswap(u);
    std::memcpy(p, &u, 4);
  }
}

// third row of an SU(3) matrix from the first two: conj(row0 x row1)
void third_row(double* m) {  // m: 9 complex as 18 doubles, rows 0 and 1 set
  auto re = [&](int r, int c) { return m[2 * (3 * r + c)]; };
  auto im = [&](int r, int c) { return m[2 * (3 * r + c) + 1]; };
  for (int c = 0; c < 3; ++c) {
    const int a = (c + 1) % 3, b = (c + 2) % 3;
    // (row0_a row1_b - row0_b row1_a), then conjugated
    const double xr = re(0, a) * re(1, b) - im(0, a) * im(1, b) - (re(0, b) * re(1, a) - im(0, b) * im(1, a));
    const double xi = re(0, a) * im(1, b) + im(0, a) * re(1, b) - (re(0, b) * im(1, a) + im(0, b) * re(1, a));
    m[2 * (6 + c)] = xr;
    m[2 * (6 + c) + 1] = -xi;
  }
}

// average plaquette and link trace on the host (file headers)
void host_plaquette(const int L[4], const double* U, double* plaq, double* ltrace) {
  const int64_t V = (int64_t)L[0] * L[1] * L[2] * L[3];
  double ps = 0.0, ts = 0.0;
  auto at = [&](int64_t site, int mu, int a, int b, int part) { return U[(((site * 4 + mu) * 3 + a) * 3 + b) * 2 + part]; };
  for (int64_t s = 0; s < V; ++s) {
    int c[4];
    int64_t t = s;
    for (int k = 0; k < 4; ++k) {
      c[k] = (int)(t % L[k]);
      t /= L[k];
    }
    auto shift = [&](int mu) {
      int cc[4] = {c[0], c[1], c[2], c[3]};
      cc[mu] = (cc[mu] + 1) % L[mu];
      return (((int64_t)cc[3] * L[2] + cc[2]) * L[1] + cc[1]) * L[0] + cc[0];
    };
    for (int mu = 0; mu < 4; ++mu) {
      ts += at(s, mu, 0, 0, 0) + at(s, mu, 1, 1, 0) + at(s, mu, 2, 2, 0);
      const int64_t xm = shift(mu);
      for (int nu = mu + 1; nu < 4; ++nu) {
        const int64_t xn = shift(nu);
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) {
            double ar = 0, ai = 0, br = 0, bi = 0;
            for (int k = 0; k < 3; ++k) {
              ar += at(s, mu, a, k, 0) * at(xm, nu, k, b, 0) - at(s, mu, a, k, 1) * at(xm, nu, k, b, 1);
              ai += at(s, mu, a, k, 0) * at(xm, nu, k, b, 1) + at(s, mu, a, k, 1) * at(xm, nu, k, b, 0);
              br += at(s, nu, a, k, 0) * at(xn, mu, k, b, 0) - at(s, nu, a, k, 1) * at(xn, mu, k, b, 1);
              bi += at(s, nu, a, k, 0) * at(xn, mu, k, b, 1) + at(s, nu, a, k, 1) * at(xn, mu, k, b, 0);
            }
            ps += ar * br + ai * bi;
          }
      }
    }
  }
  *plaq = ps / (3.0 * 6.0 * (double)V);
  *ltrace = ts / (3.0 * 4.0 * (double)V);
}

std::string trim(const std::string& s) {
  const size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

}  // namespace gio

// average plaquette and link trace (partial sums per site, reduced on the host)
__global__ void plaquette_kernel(const double2* __restrict__ U, int L0, int L1, int L2, int L3,
                                 double* __restrict__ psum, double* __restrict__ tsum) {
  const int L[4] = {L0, L1, L2, L3};
  const int64_t V = (int64_t)L0 * L1 * L2 * L3;
  double p = 0.0, tr = 0.0;
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < V; s += (int64_t)gridDim.x * blockDim.x) {
    int c[4];
    int64_t t = s;
    for (int k = 0; k < 4; ++k) {
      c[k] = (int)(t % L[k]);
      t /= L[k];
    }
    auto shift = [&](int mu) {
      int cc[4] = {c[0], c[1], c[2], c[3]};
      cc[mu] = (cc[mu] + 1) % L[mu];
      return ((int64_t)cc[3] * L2 + cc[2]) * ((int64_t)L1 * L0) + (int64_t)cc[1] * L0 + cc[0];
    };
    auto link = [&](int64_t site, int mu, int a, int b) { return U[((site * 4 + mu) * 3 + a) * 3 + b]; };
    for (int mu = 0; mu < 4; ++mu) {
      tr += link(s, mu, 0, 0).x + link(s, mu, 1, 1).x + link(s, mu, 2, 2).x;
      const int64_t xm = shift(mu);
      for (int nu = mu + 1; nu < 4; ++nu) {
        const int64_t xn = shift(nu);
        // A = U_mu(x) U_nu(x+mu); B = U_nu(x) U_mu(x+nu); Re tr(A B^dag)
        double2 A[3][3], B[3][3];
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) {
            double2 sa = make_double2(0, 0), sb = make_double2(0, 0);
            for (int k = 0; k < 3; ++k) {
              const double2 u1 = link(s, mu, a, k), u2 = link(xm, nu, k, b);
              sa.x += u1.x * u2.x - u1.y * u2.y;
              sa.y += u1.x * u2.y + u1.y * u2.x;
              const double2 v1 = link(s, nu, a, k), v2 = link(xn, mu, k, b);
              sb.x += v1.x * v2.x - v1.y * v2.y;
              sb.y += v1.x * v2.y + v1.y * v2.x;
            }
            A[a][b] = sa;
            B[a][b] = sb;
          }
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) p += A[a][b].x * B[a][b].x + A[a][b].y * B[a][b].y;
      }
    }
  }
  // block reduction
  __shared__ double sp[256], st[256];
  sp[threadIdx.x] = p;
  st[threadIdx.x] = tr;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      sp[threadIdx.x] += sp[threadIdx.x + o];
      st[threadIdx.x] += st[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    psum[blockIdx.x] = sp[0];
    tsum[blockIdx.x] = st[0];
  }
}

static gmg_status plaquette(const int dims[4], const double* U, int on_device, double* plaq, double* ltrace,
                            cudaStream_t s) {
  const int64_t V = (int64_t)dims[0] * dims[1] * dims[2] * dims[3];
  const size_t bytes = sizeof(double2) * 36 * (size_t)V;
  DevBuf tmp, part;
  const double2* Ud = reinterpret_cast<const double2*>(U);
  if (!on_device) {
    GMG_TRY(tmp.alloc(bytes));
    GMG_CUDA(cudaMemcpyAsync(tmp.p, U, bytes, cudaMemcpyHostToDevice, s));
    Ud = tmp.as<double2>();
  }
  const int grid = (int)std::min<int64_t>((V + 255) / 256, 148 * 8);
  GMG_TRY(part.alloc(sizeof(double) * 2 * grid));
  plaquette_kernel<<<grid, 256, 0, s>>>(Ud, dims[0], dims[1], dims[2], dims[3], part.as<double>(),
                                        part.as<double>() + grid);
  GMG_CUDA(cudaGetLastError());
  std::vector<double> h(2 * grid);
  GMG_CUDA(cudaMemcpyAsync(h.data(), part.p, sizeof(double) * 2 * grid, cudaMemcpyDeviceToHost, s));
  GMG_CUDA(cudaStreamSynchronize(s));
  double ps = 0.0, ts = 0.0;
  for (int k = 0; k < grid; ++k) {
    ps += h[k];
    ts += h[grid + k];
  }
  if (plaq) *plaq = ps / (3.0 * 6.0 * (double)V);
  if (ltrace) *ltrace = ts / (3.0 * 4.0 * (double)V);
  return GMG_OK;
}

}  // namespace gmg

using namespace gmg;

extern "C" gmg_status gmg_gauge_plaquette(const int dims[4], const double* U, int on_device, double* plaq,
                                          double* link_trace, gmg_stream s) {
  GMG_CHECK(dims && U, GMG_ERR_ARGUMENT, "gmg_gauge_plaquette: null argument");
  for (int k = 0; k < 4; ++k) GMG_CHECK(dims[k] >= 1, GMG_ERR_ARGUMENT, "gmg_gauge_plaquette: bad extent");
  return plaquette(dims, U, on_device, plaq, link_trace, S(s));
}

extern "C" gmg_status gmg_gauge_read_nersc(const char* path, gmg_gauge_info* info, double* U, int verify) {
  GMG_CHECK(path && info, GMG_ERR_ARGUMENT, "gmg_gauge_read_nersc: null argument");
  std::ifstream f(path, std::ios::binary);
  GMG_CHECK(f.good(), GMG_ERR_ARGUMENT, std::string("gmg_gauge_read_nersc: cannot open ") + path);
  std::memset(info, 0, sizeof(*info));
  std::string line, dtype, fp;
  bool begun = false, ended = false, have_csum = false;
  std::map<std::string, std::string> kv;
  while (std::getline(f, line)) {
    const std::string t = gio::trim(line);
    if (!begun) {
      GMG_CHECK(t == "BEGIN_HEADER", GMG_ERR_SHAPE, "gmg_gauge_read_nersc: no BEGIN_HEADER line");
      begun = true;
      continue;
    }
    if (t == "END_HEADER") {
      ended = true;
      break;
    }
    const size_t eq = t.find('=');
    if (eq == std::string::npos) continue;
    kv[gio::trim(t.substr(0, eq))] = gio::trim(t.substr(eq + 1));
  }
  GMG_CHECK(ended, GMG_ERR_SHAPE, "gmg_gauge_read_nersc: no END_HEADER line");
  for (int k = 0; k < 4; ++k) {
    auto it = kv.find("DIMENSION_" + std::to_string(k + 1));
    GMG_CHECK(it != kv.end(), GMG_ERR_SHAPE, "gmg_gauge_read_nersc: missing DIMENSION_" + std::to_string(k + 1));
    info->dims[k] = std::atoi(it->second.c_str());
    GMG_CHECK(info->dims[k] >= 1, GMG_ERR_SHAPE, "gmg_gauge_read_nersc: bad extent");
  }
  dtype = kv.count("DATATYPE") ? kv["DATATYPE"] : "";
  GMG_CHECK(dtype == "4D_SU3_GAUGE" || dtype == "4D_SU3_GAUGE_3x3", GMG_ERR_UNSUPPORTED,
            "gmg_gauge_read_nersc: DATATYPE must be 4D_SU3_GAUGE or 4D_SU3_GAUGE_3x3, got '" + dtype + "'");
  info->two_row = dtype == "4D_SU3_GAUGE";
  fp = kv.count("FLOATING_POINT") ? kv["FLOATING_POINT"] : "IEEE64BIG";
  if (fp == "IEEE64BIG" || fp == "IEEE64") {
    info->precision = 64;
    info->big_endian = 1;
  } else if (fp == "IEEE32BIG" || fp == "IEEE32") {
    info->precision = 32;
    info->big_endian = 1;
  } else if (fp == "IEEE64LITTLE") {
    info->precision = 64;
  } else if (fp == "IEEE32LITTLE") {
    info->precision = 32;
  } else {
    return fail(GMG_ERR_UNSUPPORTED, "gmg_gauge_read_nersc: unknown FLOATING_POINT '" + fp + "'");
  }
  if (kv.count("PLAQUETTE")) info->plaquette = std::atof(kv["PLAQUETTE"].c_str());
  if (kv.count("LINK_TRACE")) info->link_trace = std::atof(kv["LINK_TRACE"].c_str());
  if (kv.count("CHECKSUM")) {
    info->checksum = (uint32_t)std::strtoul(kv["CHECKSUM"].c_str(), nullptr, 16);
    have_csum = true;
  }
  if (!U) return GMG_OK;
  const int64_t V = (int64_t)info->dims[0] * info->dims[1] * info->dims[2] * info->dims[3];
  const int rows = info->two_row ? 2 : 3, wb = info->precision / 8;
  const size_t per_link = (size_t)rows * 3 * 2 * wb, bytes = per_link * 4 * (size_t)V;
  std::vector<unsigned char> buf(bytes);
  f.read(reinterpret_cast<char*>(buf.data()), (std::streamsize)bytes);
  GMG_CHECK((size_t)f.gcount() == bytes, GMG_ERR_SHAPE, "gmg_gauge_read_nersc: file shorter than its header says");
  info->checksum_data = gio::word_sum(buf.data(), bytes, info->big_endian != 0);
  for (int64_t l = 0; l < 4 * V; ++l) {
    double* m = U + 18 * l;
    const unsigned char* p = buf.data() + per_link * l;
    for (int k = 0; k < rows * 6; ++k) m[k] = gio::read_real(p + (size_t)k * wb, info->precision, info->big_endian);
    if (info->two_row) gio::third_row(m);
  }
  if (verify) {
    GMG_CHECK(!have_csum || info->checksum == info->checksum_data, GMG_ERR_NONFINITE,
              "gmg_gauge_read_nersc: checksum mismatch");
    double pl = 0.0, lt = 0.0;
    gio::host_plaquette(info->dims, U, &pl, &lt);
    const double tol = info->precision == 32 ? 1e-6 : 1e-10;
    GMG_CHECK(!kv.count("PLAQUETTE") || std::fabs(pl - info->plaquette) <= tol, GMG_ERR_NONFINITE,
              "gmg_gauge_read_nersc: plaquette differs from the header");
    GMG_CHECK(!kv.count("LINK_TRACE") || std::fabs(lt - info->link_trace) <= tol, GMG_ERR_NONFINITE,
              "gmg_gauge_read_nersc: link trace differs from the header");
  }
  return GMG_OK;
}

extern "C" gmg_status gmg_gauge_write_nersc(const char* path, const int dims[4], const double* U, int two_row,
                                           int precision, const char* ensemble_id, int sequence_number) {
  GMG_CHECK(path && dims && U, GMG_ERR_ARGUMENT, "gmg_gauge_write_nersc: null argument");
  GMG_CHECK(precision == 32 || precision == 64, GMG_ERR_ARGUMENT, "gmg_gauge_write_nersc: precision must be 32 or 64");
  for (int k = 0; k < 4; ++k) GMG_CHECK(dims[k] >= 1, GMG_ERR_ARGUMENT, "gmg_gauge_write_nersc: bad extent");
  const int64_t V = (int64_t)dims[0] * dims[1] * dims[2] * dims[3];
  const int rows = two_row ? 2 : 3, wb = precision / 8;
  const size_t per_link = (size_t)rows * 3 * 2 * wb, bytes = per_link * 4 * (size_t)V;
  std::vector<unsigned char> buf(bytes);
  for (int64_t l = 0; l < 4 * V; ++l)
    for (int k = 0; k < rows * 6; ++k)
      gio::write_real(buf.data() + per_link * l + (size_t)k * wb, U[18 * l + k], precision, true);
  double pl = 0.0, lt = 0.0;
  gio::host_plaquette(dims, U, &pl, &lt);
  std::ostringstream h;
  h.precision(12);
  char csum[16];
  std::snprintf(csum, sizeof(csum), "%x", gio::word_sum(buf.data(), bytes, true));
  char date[64];
  const std::time_t now = std::time(nullptr);
  std::strftime(date, sizeof(date), "%a %b %d %H:%M:%S %Y", std::gmtime(&now));
  h << "BEGIN_HEADER\n"
    << "HDR_VERSION = 1.0\n"
    << "DATATYPE = " << (two_row ? "4D_SU3_GAUGE" : "4D_SU3_GAUGE_3x3") << "\n"
    << "STORAGE_FORMAT = 1.0\n";
  for (int k = 0; k < 4; ++k) h << "DIMENSION_" << k + 1 << " = " << dims[k] << "\n";
  h << "LINK_TRACE = " << lt << "\n"
    << "PLAQUETTE = " << pl << "\n";
  for (int k = 0; k < 4; ++k) h << "BOUNDARY_" << k + 1 << " = PERIODIC\n";
  h << "CHECKSUM = " << csum << "\n"
    << "ENSEMBLE_ID = " << (ensemble_id ? ensemble_id : "unknown") << "\n"
    << "ENSEMBLE_LABEL = unknown\n"
    << "SEQUENCE_NUMBER = " << sequence_number << "\n"
    << "CREATOR = libgmg_b200\n"
    << "CREATION_DATE = " << date << "\n"
    << "FLOATING_POINT = " << (precision == 64 ? "IEEE64BIG" : "IEEE32BIG") << "\n"
    << "END_HEADER\n";
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  GMG_CHECK(f.good(), GMG_ERR_ARGUMENT, std::string("gmg_gauge_write_nersc: cannot create ") + path);
  const std::string hs = h.str();
  f.write(hs.data(), (std::streamsize)hs.size());
  f.write(reinterpret_cast<const char*>(buf.data()), (std::streamsize)bytes);
  GMG_CHECK(f.good(), GMG_ERR_ARGUMENT, "gmg_gauge_write_nersc: write failed");
  return GMG_OK;
}

// LIME record header: magic, version, flags, payload length, type string
namespace gmg {
namespace gio {
struct LimeRecord {
  uint64_t offset = 0, length = 0;
  std::string type;
};

static bool lime_records(std::ifstream& f, std::vector<LimeRecord>& out) {
  f.seekg(0, std::ios::end);
  const uint64_t size = (uint64_t)f.tellg();
  uint64_t pos = 0;
  while (pos + 144 <= size) {
    unsigned char hd[144];
    f.seekg((std::streamoff)pos);
    f.read(reinterpret_cast<char*>(hd), 144);
    if (f.gcount() != 144) return false;
    uint32_t magic;
    std::memcpy(&magic, hd, 4);
    if (!host_big_endian()) magic = bswap(magic);
    if (magic != 0x456789abu) return false;
    uint64_t len;
    std::memcpy(&len, hd + 8, 8);
    if (!host_big_endian()) len = bswap(len);
    LimeRecord r;
    r.offset = pos + 144;
    r.length = len;
    const char* ty = reinterpret_cast<const char*>(hd + 16);
    r.type.assign(ty, strnlen(ty, 128));
    out.push_back(r);
    pos = r.offset + ((len + 7) & ~uint64_t(7));
  }
  return !out.empty();
}

static std::string xml_field(const std::string& xml, const std::string& tag) {
  const size_t a = xml.find("<" + tag + ">");
  if (a == std::string::npos) return "";
  const size_t b = xml.find("</" + tag + ">", a);
  if (b == std::string::npos) return "";
  return trim(xml.substr(a + tag.size() + 2, b - a - tag.size() - 2));
}
}  // namespace gio
}  // namespace gmg

extern "C" gmg_status gmg_gauge_read_ildg(const char* path, gmg_gauge_info* info, double* U) {
  GMG_CHECK(path && info, GMG_ERR_ARGUMENT, "gmg_gauge_read_ildg: null argument");
  std::ifstream f(path, std::ios::binary);
  GMG_CHECK(f.good(), GMG_ERR_ARGUMENT, std::string("gmg_gauge_read_ildg: cannot open ") + path);
  std::memset(info, 0, sizeof(*info));
  std::vector<gio::LimeRecord> recs;
  GMG_CHECK(gio::lime_records(f, recs), GMG_ERR_SHAPE, "gmg_gauge_read_ildg: not a LIME file");
  const gio::LimeRecord *fmt = nullptr, *bin = nullptr;
  for (const auto& r : recs) {
    if (r.type == "ildg-format") fmt = &r;
    if (r.type == "ildg-binary-data") bin = &r;
  }
  GMG_CHECK(fmt && bin, GMG_ERR_SHAPE, "gmg_gauge_read_ildg: no ildg-format / ildg-binary-data record");
  f.clear();
  f.seekg((std::streamoff)fmt->offset);
  std::string xml(fmt->length, '\0');
  f.read(&xml[0], (std::streamsize)fmt->length);
  info->precision = std::atoi(gio::xml_field(xml, "precision").c_str());
  GMG_CHECK(info->precision == 32 || info->precision == 64, GMG_ERR_UNSUPPORTED,
            "gmg_gauge_read_ildg: precision must be 32 or 64");
  const char* tags[4] = {"lx", "ly", "lz", "lt"};
  for (int k = 0; k < 4; ++k) {
    info->dims[k] = std::atoi(gio::xml_field(xml, tags[k]).c_str());
    GMG_CHECK(info->dims[k] >= 1, GMG_ERR_SHAPE, "gmg_gauge_read_ildg: bad lattice extent");
  }
  info->big_endian = 1;
  if (!U) return GMG_OK;
  const int64_t V = (int64_t)info->dims[0] * info->dims[1] * info->dims[2] * info->dims[3];
  const int wb = info->precision / 8;
  const size_t bytes = (size_t)V * 4 * 18 * wb;
  GMG_CHECK(bin->length == bytes, GMG_ERR_SHAPE, "gmg_gauge_read_ildg: binary record size differs from the format");
  std::vector<unsigned char> buf(bytes);
  f.clear();
  f.seekg((std::streamoff)bin->offset);
  f.read(reinterpret_cast<char*>(buf.data()), (std::streamsize)bytes);
  GMG_CHECK((size_t)f.gcount() == bytes, GMG_ERR_SHAPE, "gmg_gauge_read_ildg: file truncated");
  for (size_t k = 0; k < (size_t)V * 4 * 18; ++k) U[k] = gio::read_real(buf.data() + k * wb, info->precision, true);
  return GMG_OK;
}
