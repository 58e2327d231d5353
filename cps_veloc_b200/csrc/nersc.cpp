// NERSC gauge-configuration archives, as the reference reads and writes
// them (ReadLatticeParallel::read, ReadLatticePar.C; WriteLatticeParallel::
// write, WriteLatticePar.C; LatticeHeader, latheader.C:195-310; FPConv,
// fpconv.C:279-395):
//
//   BEGIN_HEADER / KEY = value lines / END_HEADER, then for every site in
//   lexicographic order (x fastest, t slowest) the four links mu = 0..3,
//   each either its first two rows (DATATYPE = 4D_SU3_GAUGE, 12 reals) or
//   the whole matrix (4D_SU3_GAUGE_3x3, 18 reals), row-major, (re, im), in
//   the FLOATING_POINT format (IEEE32[BIG|LITTLE], IEEE64[BIG|LITTLE];
//   IEEE32 / IEEE64 are big-endian).
//   CHECKSUM: the sum modulo 2^32 of the data as 32-bit words in host order
//   (an 8-byte value contributes its two halves).
//   PLAQUETTE = SumReTrPlaq / (18 V), LINK_TRACE = sum Re tr U / (12 V).
//
// The reference parses the header with a "key = value" map that trims
// spaces (latheader.C:33-55) and reads PLAQUETTE / LINK_TRACE with %f; the
// reader here does the same.  On reading, a stored two-row link gets its
// third row as conj(row0 x row1) with the reference's operand order
// (ReadLatticePar.C, recon_row_3).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <thread>
#include <unistd.h>
#include <vector>

#include "../../include/cpsgpu.h"
#include "cpsgpu_impl.h"

namespace cpsgpu {

namespace {

// FP_FORMAT names in the reference's enum order (fpconv.C:12-22)
const char *const FP_NAMES[] = {"n/a", "AUTOMATIC", "TIDSP32", "IEEE32", "IEEE32BIG", "IEEE32LITTLE",
                                "IEEE64", "IEEE64BIG", "IEEE64LITTLE"};

int fp_size(int f) {
  if (f == CPSGPU_FP_IEEE32 || f == CPSGPU_FP_IEEE32BIG || f == CPSGPU_FP_IEEE32LITTLE) return 4;
  if (f == CPSGPU_FP_IEEE64 || f == CPSGPU_FP_IEEE64BIG || f == CPSGPU_FP_IEEE64LITTLE) return 8;
  return 0;
}
bool fp_big(int f) {
  return f == CPSGPU_FP_IEEE32 || f == CPSGPU_FP_IEEE32BIG || f == CPSGPU_FP_IEEE64 || f == CPSGPU_FP_IEEE64BIG;
}

std::string trim(const std::string &s) {
  const size_t a = s.find_first_not_of(" \r\t"), b = s.find_last_not_of(" \r\t");
  if (a == std::string::npos) return "";
  return s.substr(a, b - a + 1);
}

void check_dims(const int node_sites[4]) {
  if (!node_sites) throw Error(CPSGPU_ERR_ARG, "null node_sites");
  for (int k = 0; k < 4; k++)
    if (node_sites[k] < 1) throw Error(CPSGPU_ERR_ARG, "bad lattice extent");
}

// value of file word k (fp bytes, file endianness) as a double
double load_value(const unsigned char *p, int size, bool big) {
  unsigned char b[8];
  for (int k = 0; k < size; k++) b[k] = big ? p[size - 1 - k] : p[k];  // to little-endian (host)
  if (size == 8) {
    double d;
    std::memcpy(&d, b, 8);
    return d;
  }
  float f;
  std::memcpy(&f, b, 4);
  return (double)f;
}

void store_value(unsigned char *p, int size, bool big, double v) {
  unsigned char b[8];
  if (size == 8) std::memcpy(b, &v, 8);
  else {
    const float f = (float)v;
    std::memcpy(b, &f, 4);
  }
  for (int k = 0; k < size; k++) p[k] = big ? b[size - 1 - k] : b[k];
}

// FPConv::checksum: 32-bit words of the data in host (little-endian) order
uint32_t checksum32(const unsigned char *data, size_t nbytes, bool big) {
  uint32_t s = 0;
  for (size_t o = 0; o + 4 <= nbytes; o += 4) {
    const unsigned char *p = data + o;
    const uint32_t w = big ? ((uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3])
                           : ((uint32_t)p[3] << 24 | (uint32_t)p[2] << 16 | (uint32_t)p[1] << 8 | p[0]);
    s += w;
  }
  return s;
}

// third row of a row-major link from its first two (ReadLatticePar.C)
void reconstruct_row3(double *rec) {
  rec[12] = rec[2] * rec[10] - rec[3] * rec[11] - rec[4] * rec[8] + rec[5] * rec[9];
  rec[13] = -rec[2] * rec[11] - rec[3] * rec[10] + rec[4] * rec[9] + rec[5] * rec[8];
  rec[14] = -rec[0] * rec[10] + rec[1] * rec[11] + rec[4] * rec[6] - rec[5] * rec[7];
  rec[15] = rec[0] * rec[11] + rec[1] * rec[10] - rec[4] * rec[7] - rec[5] * rec[6];
  rec[16] = rec[0] * rec[8] - rec[1] * rec[9] - rec[2] * rec[6] + rec[3] * rec[7];
  rec[17] = -rec[0] * rec[9] - rec[1] * rec[8] + rec[2] * rec[7] + rec[3] * rec[6];
}

void copy_field(char *dst, size_t n, const std::string &s) {
  std::snprintf(dst, n, "%s", s.c_str());
}

std::string fmt10(double v) {
  char b[64];
  std::snprintf(b, sizeof b, "%.10g", v);
  return b;
}

}  // namespace

// SumReTrPlaq and the link-trace sum of a CANONICAL host field (the writer's
// header values; Lattice::SumReTrPlaqNode, lattice_base.C:2878)
void host_gauge_sums(const int L[4], const double *u, double *sum_plaq, double *sum_link) {
  const long vol = (long)L[0] * L[1] * L[2] * L[3];
  auto lex = [&](int x, int y, int z, int t) { return x + (long)L[0] * (y + (long)L[1] * (z + (long)L[2] * t)); };
  const unsigned nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<double> ps(nth, 0.0), ls(nth, 0.0);
  auto work = [&](unsigned id) {
    double sp = 0.0, sl = 0.0;
    for (long s = id; s < vol; s += nth) {
      int c[4];
      long r = s;
      for (int k = 0; k < 4; k++) {
        c[k] = (int)(r % L[k]);
        r /= L[k];
      }
      const double *us = u + 72 * s;
      for (int mu = 0; mu < 4; mu++) sl += us[18 * mu] + us[18 * mu + 8] + us[18 * mu + 16];
      for (int mu = 0; mu < 3; mu++)
        for (int nu = mu + 1; nu < 4; nu++) {
          int cm[4] = {c[0], c[1], c[2], c[3]}, cn[4] = {c[0], c[1], c[2], c[3]};
          cm[mu] = (cm[mu] + 1) % L[mu];
          cn[nu] = (cn[nu] + 1) % L[nu];
          const double *a = us + 18 * mu, *b = u + 72 * lex(cm[0], cm[1], cm[2], cm[3]) + 18 * nu;
          const double *d = us + 18 * nu, *e = u + 72 * lex(cn[0], cn[1], cn[2], cn[3]) + 18 * mu;
          // Re tr[(a b)(d e)^dag]
          double m1[18], m2[18];
          for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
              double r1 = 0, i1 = 0, r2 = 0, i2 = 0;
              for (int k = 0; k < 3; k++) {
                const double *pa = a + 2 * (3 * i + k), *pb = b + 2 * (3 * k + j);
                const double *pd = d + 2 * (3 * i + k), *pe = e + 2 * (3 * k + j);
                r1 += pa[0] * pb[0] - pa[1] * pb[1];
                i1 += pa[0] * pb[1] + pa[1] * pb[0];
                r2 += pd[0] * pe[0] - pd[1] * pe[1];
                i2 += pd[0] * pe[1] + pd[1] * pe[0];
              }
              m1[2 * (3 * i + j)] = r1;
              m1[2 * (3 * i + j) + 1] = i1;
              m2[2 * (3 * i + j)] = r2;
              m2[2 * (3 * i + j) + 1] = i2;
            }
          for (int k = 0; k < 18; k++) sp += m1[k] * m2[k];
        }
    }
    ps[id] = sp;
    ls[id] = sl;
  };
  std::vector<std::thread> th;
  for (unsigned k = 0; k < nth; k++) th.emplace_back(work, k);
  for (auto &t : th) t.join();
  double a = 0.0, b = 0.0;
  for (unsigned k = 0; k < nth; k++) {
    a += ps[k];
    b += ls[k];
  }
  if (sum_plaq) *sum_plaq = a;
  if (sum_link) *sum_link = b;
}

void nersc_read(const char *path, const int node_sites[4], double *u, cpsgpu_nersc_header *hdr) {
  check_dims(node_sites);
  if (!path || !u) throw Error(CPSGPU_ERR_ARG, "null argument");
  std::ifstream in(path, std::ios::binary);
  if (!in.good()) throw Error(CPSGPU_ERR_ARG, std::string("cannot open ") + path);
  std::map<std::string, std::string> h;
  std::string line;
  bool end = false;
  while (std::getline(in, line)) {
    if (line.find("END_HEADER") != std::string::npos) {
      end = true;
      break;
    }
    const size_t eq = line.find('=');
    if (eq != std::string::npos && eq > 0) h.emplace(trim(line.substr(0, eq)), trim(line.substr(eq + 1)));
  }
  if (!end) throw Error(CPSGPU_ERR_ARG, "no END_HEADER");
  auto get = [&](const char *k) -> std::string {
    auto it = h.find(k);
    return it == h.end() ? std::string() : it->second;
  };
  const bool recon = get("DATATYPE") == "4D_SU3_GAUGE";
  if (!recon && get("DATATYPE") != "4D_SU3_GAUGE_3x3")
    throw Error(CPSGPU_ERR_ARG, "DATATYPE must be 4D_SU3_GAUGE or 4D_SU3_GAUGE_3x3");
  int dims[4];
  for (int k = 0; k < 4; k++) {
    char key[16];
    std::snprintf(key, sizeof key, "DIMENSION_%d", k + 1);
    dims[k] = std::atoi(get(key).c_str());
    if (dims[k] != node_sites[k]) throw Error(CPSGPU_ERR_ARG, "lattice dimensions differ from the header");
  }
  int fmt = 0;
  const std::string fpn = get("FLOATING_POINT");
  for (int k = 1; k < 9; k++)
    if (fpn == FP_NAMES[k]) fmt = k;
  const int size = fp_size(fmt);
  if (!size) throw Error(CPSGPU_ERR_ARG, "FLOATING_POINT format not recognised: " + fpn);
  unsigned int csum_hdr = 0;
  std::sscanf(get("CHECKSUM").c_str(), "%x", &csum_hdr);
  float plaq_f = 0.f, ltr_f = 0.f;
  std::sscanf(get("PLAQUETTE").c_str(), "%f", &plaq_f);
  std::sscanf(get("LINK_TRACE").c_str(), "%f", &ltr_f);

  const long vol = (long)node_sites[0] * node_sites[1] * node_sites[2] * node_sites[3];
  const int per = recon ? 12 : 18;
  const size_t nbytes = (size_t)vol * 4 * per * size;
  std::vector<unsigned char> buf(nbytes);
  in.read(reinterpret_cast<char *>(buf.data()), (std::streamsize)nbytes);
  if ((size_t)in.gcount() != nbytes) throw Error(CPSGPU_ERR_ARG, "file shorter than the lattice");
  const bool big = fp_big(fmt);
  const uint32_t csum = checksum32(buf.data(), nbytes, big);
  if (csum != csum_hdr) {
    char msg[96];
    std::snprintf(msg, sizeof msg, "checksum error: header %x, data %x", csum_hdr, csum);
    throw Error(CPSGPU_ERR_ARG, msg);
  }
  for (long l = 0; l < vol * 4; l++) {
    double *rec = u + 18 * l;
    const unsigned char *src = buf.data() + (size_t)l * per * size;
    for (int k = 0; k < per; k++) rec[k] = load_value(src + (size_t)k * size, size, big);
    if (recon) reconstruct_row3(rec);
  }
  if (hdr) {
    std::memset(hdr, 0, sizeof(*hdr));
    for (int k = 0; k < 4; k++) hdr->dims[k] = dims[k];
    hdr->recon_row_3 = recon ? 1 : 0;
    hdr->fp_format = fmt;
    hdr->plaquette = plaq_f;
    hdr->link_trace = ltr_f;
    hdr->checksum = csum_hdr;
    hdr->sequence_number = std::atoi(get("SEQUENCE_NUMBER").c_str());
    copy_field(hdr->ensemble_id, sizeof hdr->ensemble_id, get("ENSEMBLE_ID"));
    copy_field(hdr->ensemble_label, sizeof hdr->ensemble_label, get("ENSEMBLE_LABEL"));
    copy_field(hdr->creator, sizeof hdr->creator, get("CREATOR"));
  }
}

void nersc_write(const char *path, const int node_sites[4], const double *u, int recon_row_3, int fp_format,
                 const cpsgpu_nersc_header *meta, cpsgpu_nersc_header *out) {
  check_dims(node_sites);
  if (!path || !u) throw Error(CPSGPU_ERR_ARG, "null argument");
  const int size = fp_size(fp_format);
  if (!size) throw Error(CPSGPU_ERR_ARG, "fp_format must be one of the IEEE32 / IEEE64 formats");
  const bool big = fp_big(fp_format);
  const long vol = (long)node_sites[0] * node_sites[1] * node_sites[2] * node_sites[3];
  double sp = 0.0, sl = 0.0;
  host_gauge_sums(node_sites, u, &sp, &sl);
  const double plaq = sp / (18.0 * (double)vol), ltrace = sl / (12.0 * (double)vol);
  const int per = recon_row_3 ? 12 : 18;
  const size_t nbytes = (size_t)vol * 4 * per * size;
  std::vector<unsigned char> buf(nbytes);
  for (long l = 0; l < vol * 4; l++)
    for (int k = 0; k < per; k++) store_value(buf.data() + ((size_t)l * per + k) * size, size, big, u[18 * l + k]);
  const uint32_t csum = checksum32(buf.data(), nbytes, big);

  char host[256] = {0};
  gethostname(host, sizeof host - 1);
  const std::time_t now = std::time(nullptr);
  std::string date = std::asctime(std::localtime(&now));
  while (!date.empty() && (date.back() == '\n' || date.back() == '\r')) date.pop_back();
  std::ostringstream o;
  o << "BEGIN_HEADER\n";
  o << "HDR_VERSION = 1.0\n";
  o << "DATATYPE = " << (recon_row_3 ? "4D_SU3_GAUGE" : "4D_SU3_GAUGE_3x3") << "\n";
  o << "STORAGE_FORMAT = 1.0\n";
  for (int k = 0; k < 4; k++) o << "DIMENSION_" << k + 1 << " = " << node_sites[k] << "\n";
  o << "LINK_TRACE = " << fmt10(ltrace) << "\n";
  o << "PLAQUETTE  = " << fmt10(plaq) << "\n";
  for (int k = 0; k < 4; k++) o << "BOUNDARY_" << k + 1 << " = PERIODIC\n";
  char cs[16];
  std::snprintf(cs, sizeof cs, "%8x", csum);
  o << "CHECKSUM = " << cs << "\n";
  o << "ENSEMBLE_ID = " << (meta ? meta->ensemble_id : "") << "\n";
  o << "ENSEMBLE_LABEL = " << (meta ? meta->ensemble_label : "") << "\n";
  o << "SEQUENCE_NUMBER = " << (meta ? meta->sequence_number : 0) << "\n";
  o << "CREATOR = " << (meta && meta->creator[0] ? meta->creator : "cps_veloc_b200") << "\n";
  o << "CREATOR_HARDWARE = " << host << "\n";
  o << "CREATION_DATE = " << date << "\n";
  o << "ARCHIVE_DATE = " << date << "\n";
  o << "FLOATING_POINT = " << FP_NAMES[fp_format] << "\n";
  o << "END_HEADER\n";
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f.good()) throw Error(CPSGPU_ERR_ARG, std::string("cannot open ") + path + " for writing");
  const std::string hs = o.str();
  f.write(hs.data(), (std::streamsize)hs.size());
  f.write(reinterpret_cast<const char *>(buf.data()), (std::streamsize)nbytes);
  if (!f.good()) throw Error(CPSGPU_ERR_ARG, "write failed");
  if (out) {
    std::memset(out, 0, sizeof(*out));
    for (int k = 0; k < 4; k++) out->dims[k] = node_sites[k];
    out->recon_row_3 = recon_row_3 ? 1 : 0;
    out->fp_format = fp_format;
    out->plaquette = plaq;
    out->link_trace = ltrace;
    out->checksum = csum;
  }
}

}  // namespace cpsgpu
