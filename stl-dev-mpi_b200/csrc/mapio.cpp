// Map files: NESTED .npy and HEALPix FITS binary tables (mapio.hpp).
// The formats are those of the reference's io.rs (crates/stl-mpi/src/io.rs):
// .npy version 1-3 headers with '<f8' '>f8' '<f4' '>f4' '<i8' '>i8' '<i4'
// '>i4' arrays in C order; FITS files of 2880-byte blocks whose first
// binary table holds the map in its first column ('E' or 'D', a repeat
// count allowed), NESTED unless the header says ORDERING = 'RING'.
#include "mapio.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <stdexcept>

#include "healpix.cuh"

namespace stl {
namespace mapio {
namespace {

constexpr size_t kBlock = 2880;  // FITS record
constexpr size_t kCard = 80;     // FITS header card

[[noreturn]] void fail(const std::string& path, const std::string& what) {
  throw std::runtime_error(path + ": " + what);
}

bool is_fits(const std::string& path) {
  const size_t dot = path.rfind('.');
  if (dot == std::string::npos) return false;
  const std::string ext = path.substr(dot + 1);
  return ext == "fits" || ext == "fit";
}

std::ifstream open_in(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) fail(path, "cannot open for reading");
  return f;
}

// n bytes at offset (all of them, or an error)
std::vector<unsigned char> read_at(const std::string& path, uint64_t offset, size_t n) {
  std::ifstream f = open_in(path);
  std::vector<unsigned char> b(n);
  f.seekg((std::streamoff)offset);
  if (n && !f.read(reinterpret_cast<char*>(b.data()), (std::streamsize)n)) fail(path, "file shorter than its header says");
  return b;
}

bool host_little() {
  const uint16_t one = 1;
  unsigned char c;
  std::memcpy(&c, &one, 1);
  return c == 1;
}

// a value of `size` bytes in the given byte order, as the host's
template <typename V>
V load_as(const unsigned char* p, bool big) {
  unsigned char t[sizeof(V)];
  std::memcpy(t, p, sizeof(V));
  if (big == host_little()) std::reverse(t, t + sizeof(V));
  V v;
  std::memcpy(&v, t, sizeof(V));
  return v;
}

template <typename V>
void store_as(unsigned char* p, V v, bool big) {
  std::memcpy(p, &v, sizeof(V));
  if (big == host_little()) std::reverse(p, p + sizeof(V));
}

// ---- .npy ----------------------------------------------------------------------

struct Npy {
  uint64_t offset = 0;  // first data byte
  char kind = 'f';      // 'f' float, 'i' signed integer
  int size = 8;         // bytes per element
  bool big = false;     // big-endian elements
  std::vector<size_t> shape;
  size_t count = 1;
};

// the value of 'key' in the header dictionary (the text after its colon)
std::string dict_field(const std::string& dict, const std::string& key) {
  const size_t at = dict.find("'" + key + "'");
  if (at == std::string::npos) return std::string();
  size_t p = dict.find(':', at + key.size() + 2);
  if (p == std::string::npos) return std::string();
  ++p;
  while (p < dict.size() && dict[p] == ' ') ++p;
  return dict.substr(p);
}

Npy npy_layout(const std::string& path) {
  std::vector<unsigned char> head = read_at(path, 0, 12);
  if (std::memcmp(head.data(), "\x93NUMPY", 6) != 0) fail(path, "not a .npy file");
  const int major = head[6];
  size_t hlen, start;
  if (major == 1) {
    hlen = (size_t)head[8] | ((size_t)head[9] << 8);
    start = 10;
  } else if (major == 2 || major == 3) {
    hlen = (size_t)head[8] | ((size_t)head[9] << 8) | ((size_t)head[10] << 16) | ((size_t)head[11] << 24);
    start = 12;
  } else {
    fail(path, "unknown .npy version " + std::to_string(major));
  }
  const std::vector<unsigned char> text = read_at(path, start, hlen);
  const std::string dict(text.begin(), text.end());
  Npy L;
  L.offset = start + hlen;
  // descr: '<f8' and the like (a structured dtype is a list, not a string)
  const std::string descr = dict_field(dict, "descr");
  if (descr.empty() || descr[0] != '\'') fail(path, "structured arrays are not maps");
  const size_t close = descr.find('\'', 1);
  const std::string d = descr.substr(1, close == std::string::npos ? std::string::npos : close - 1);
  if (d.size() != 3) fail(path, "unsupported dtype " + d);
  if (d[0] == '>') L.big = true;
  else if (d[0] == '<' || d[0] == '|' || d[0] == '=') L.big = false;
  else fail(path, "unsupported dtype " + d);
  L.kind = d[1];
  L.size = d[2] - '0';
  if (!((L.kind == 'f' || L.kind == 'i') && (L.size == 4 || L.size == 8))) fail(path, "unsupported dtype " + d);
  if (dict_field(dict, "fortran_order").rfind("True", 0) == 0) fail(path, "Fortran-ordered arrays are not supported");
  const std::string shape = dict_field(dict, "shape");
  if (shape.empty() || shape[0] != '(') fail(path, "no shape");
  const size_t end = shape.find(')');
  if (end == std::string::npos) fail(path, "bad shape");
  std::string inner = shape.substr(1, end - 1);
  size_t p = 0;
  while (p < inner.size()) {
    size_t q = inner.find(',', p);
    if (q == std::string::npos) q = inner.size();
    std::string tok = inner.substr(p, q - p);
    tok.erase(std::remove(tok.begin(), tok.end(), ' '), tok.end());
    if (!tok.empty()) {
      for (char c : tok)
        if (c < '0' || c > '9') fail(path, "bad shape");
      L.shape.push_back((size_t)std::stoull(tok));
    }
    p = q + 1;
  }
  L.count = 1;
  for (size_t s : L.shape) L.count *= s;
  return L;
}

void npy_values(const Npy& L, const unsigned char* b, size_t n, double* out) {
  for (size_t i = 0; i < n; ++i, b += L.size) {
    if (L.kind == 'f') out[i] = L.size == 8 ? load_as<double>(b, L.big) : (double)load_as<float>(b, L.big);
    else out[i] = L.size == 8 ? (double)load_as<int64_t>(b, L.big) : (double)load_as<int32_t>(b, L.big);
  }
}

// the header of a little-endian float64 .npy of this shape, padded so that
// the data starts on a 64-byte boundary
std::string npy_header(const std::vector<size_t>& shape) {
  std::string dims;
  for (size_t s : shape) dims += std::to_string(s) + ",";
  if (shape.size() > 1) dims.pop_back();  // (n,) for one axis, (a,b) for more
  std::string h = "{'descr': '<f8', 'fortran_order': False, 'shape': (" + dims + "), }";
  while ((10 + h.size() + 1) % 64 != 0) h += ' ';
  h += '\n';
  std::string out("\x93NUMPY\x01\x00", 8);
  out += (char)(h.size() & 0xff);
  out += (char)((h.size() >> 8) & 0xff);
  return out + h;
}

// ---- FITS ----------------------------------------------------------------------

struct Fits {
  uint64_t offset = 0;  // first byte of the table's data
  size_t row = 0;       // bytes of a row (NAXIS1)
  size_t repeat = 1;    // pixels a row (TFORM1's repeat count)
  size_t width = 4;     // bytes of a pixel ('E' 4, 'D' 8)
  size_t rows = 0;      // NAXIS2
  bool nested = true;
};

// the cards of the header starting at `at` (keyword -> value: a quoted
// string without its quotes and trailing blanks, or the text before a '/'
// comment), and the header's length in whole records
struct Header {
  std::vector<std::pair<std::string, std::string>> cards;
  size_t length = 0;
  const std::string* get(const std::string& k) const {
    for (const auto& c : cards)
      if (c.first == k) return &c.second;
    return nullptr;
  }
  size_t integer(const std::string& k) const {
    const std::string* v = get(k);
    if (!v || v->empty()) return 0;
    for (char c : *v)
      if (c < '0' || c > '9') return 0;
    return (size_t)std::stoull(*v);
  }
};

std::string trim(const std::string& s) {
  const size_t a = s.find_first_not_of(' ');
  if (a == std::string::npos) return std::string();
  return s.substr(a, s.find_last_not_of(' ') - a + 1);
}

Header parse_header(std::ifstream& f, const std::string& path, uint64_t at) {
  Header h;
  char card[kCard];
  f.clear();
  f.seekg((std::streamoff)at);
  for (size_t n = 0;; ++n) {
    if (!f.read(card, kCard)) fail(path, "no binary table");
    const std::string text(card, kCard);
    const std::string key = trim(text.substr(0, 8));
    if (key == "END") {
      h.length = ((n + 1) * kCard + kBlock - 1) / kBlock * kBlock;
      return h;
    }
    if (text.compare(8, 2, "= ") != 0) continue;
    const std::string raw = trim(text.substr(10));
    std::string value;
    if (!raw.empty() && raw[0] == '\'') {
      const size_t q = raw.find('\'', 1);
      value = trim(raw.substr(1, q == std::string::npos ? std::string::npos : q - 1));
    } else {
      value = trim(raw.substr(0, raw.find('/')));
    }
    h.cards.emplace_back(key, value);
  }
}

// the first binary table of the file
Fits fits_layout(const std::string& path) {
  std::ifstream f = open_in(path);
  uint64_t at = 0;
  for (;;) {
    const Header h = parse_header(f, path, at);
    const std::string* xt = h.get("XTENSION");
    if (xt && *xt == "BINTABLE") {
      const std::string* form = h.get("TFORM1");
      if (!form) fail(path, "no TFORM1");
      size_t k = 0;
      while (k < form->size() && (*form)[k] >= '0' && (*form)[k] <= '9') ++k;
      if (k == form->size()) fail(path, "bad TFORM1");
      Fits L;
      L.repeat = k ? (size_t)std::stoull(form->substr(0, k)) : 1;
      const char code = (*form)[k];
      if (code == 'E') L.width = 4;
      else if (code == 'D') L.width = 8;
      else fail(path, std::string("column type ") + code + " is not a float map");
      L.offset = at + h.length;
      L.row = h.integer("NAXIS1");
      L.rows = h.integer("NAXIS2");
      if (L.row < L.repeat * L.width) fail(path, "row narrower than its first column");
      const std::string* ord = h.get("ORDERING");
      if (!ord || *ord == "NESTED") L.nested = true;
      else if (*ord == "RING") L.nested = false;
      else fail(path, "unknown ORDERING " + *ord);
      return L;
    }
    // skip this HDU's data: the product of its axes plus the heap, in records
    const size_t naxis = h.integer("NAXIS");
    size_t size = naxis ? 1 : 0;
    for (size_t i = 1; i <= naxis; ++i) size *= h.integer("NAXIS" + std::to_string(i));
    at += h.length + (size + h.integer("PCOUNT") + kBlock - 1) / kBlock * kBlock;
  }
}

void fits_values(const Fits& L, const unsigned char* b, size_t first_row, size_t start, size_t end, double* out) {
  for (size_t p = start; p < end; ++p) {
    const unsigned char* q = b + (p / L.repeat - first_row) * L.row + (p % L.repeat) * L.width;
    out[p - start] = L.width == 4 ? (double)load_as<float>(q, true) : load_as<double>(q, true);
  }
}

std::string card(const std::string& key, const std::string& value) {
  std::string c = key;
  c.resize(8, ' ');
  if (!value.empty()) {
    c += "= ";
    std::string v = value;
    if (v.size() < 20) v.insert(0, 20 - v.size(), ' ');  // right-justified in columns 11-30
    c += v;
  }
  c.resize(kCard, ' ');
  return c;
}

std::string quoted(const std::string& s) {
  std::string v = "'" + s;
  if (v.size() < 9) v.resize(9, ' ');  // strings padded to at least 8 characters
  v += "'";
  v.resize(std::max<size_t>(v.size(), 20), ' ');  // left-justified
  return v;
}

void pad_to_block(std::string& b, char fill) {
  if (b.size() % kBlock) b.append(kBlock - b.size() % kBlock, fill);
}

// the primary header and the table's header for n pixels
std::string fits_headers(size_t n, const std::string& column, bool dbl) {
  const int64_t nside = nside_of(n);
  std::string b;
  for (const auto& c : {card("SIMPLE", "T"), card("BITPIX", "8"), card("NAXIS", "0"), card("EXTEND", "T"),
                        card("END", "")})
    b += c;
  pad_to_block(b, ' ');
  const std::string cards[] = {
      card("XTENSION", quoted("BINTABLE")), card("BITPIX", "8"), card("NAXIS", "2"),
      card("NAXIS1", dbl ? "8" : "4"), card("NAXIS2", std::to_string(n)), card("PCOUNT", "0"), card("GCOUNT", "1"),
      card("TFIELDS", "1"), card("TTYPE1", quoted(column)), card("TFORM1", quoted(dbl ? "D" : "E")),
      card("PIXTYPE", quoted("HEALPIX")), card("ORDERING", quoted("NESTED")), card("COORDSYS", quoted("C")),
      card("EXTNAME", quoted("xtension")), card("NSIDE", std::to_string(nside)), card("FIRSTPIX", "0"),
      card("LASTPIX", std::to_string(n - 1)), card("INDXSCHM", quoted("IMPLICIT")), card("OBJECT", quoted("FULLSKY")),
      card("END", "")};
  for (const auto& c : cards) b += c;
  pad_to_block(b, ' ');
  return b;
}

void write_file(const std::string& path, const std::string& bytes) {
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) fail(path, "cannot open for writing");
  if (!f.write(bytes.data(), (std::streamsize)bytes.size())) fail(path, "write failed");
}

}  // namespace
}  // namespace mapio
}  // namespace stl

namespace stl {
namespace mapio {

int64_t nside_of(size_t npix) {
  const int64_t nside = (int64_t)std::llround(std::sqrt((double)(npix / 12)));
  if (nside < 1 || (size_t)(12 * nside * nside) != npix || (nside & (nside - 1)) != 0)
    throw std::runtime_error(std::to_string(npix) + " pixels is not a full-sky HEALPix map");
  return nside;
}

size_t map_len(const std::string& path) {
  if (is_fits(path)) {
    const Fits L = fits_layout(path);
    return L.repeat * L.rows;
  }
  return npy_layout(path).count;
}

std::vector<size_t> npy_shape(const std::string& path) { return npy_layout(path).shape; }

std::vector<double> read_npy(const std::string& path, std::vector<size_t>* shape) {
  const Npy L = npy_layout(path);
  const std::vector<unsigned char> b = read_at(path, L.offset, L.count * L.size);
  std::vector<double> out(L.count);
  npy_values(L, b.data(), L.count, out.data());
  if (shape) *shape = L.shape;
  return out;
}

namespace {
// the values of a FITS map in file order
std::vector<double> fits_all(const std::string& path, const Fits& L) {
  const size_t n = L.repeat * L.rows;
  const std::vector<unsigned char> b = read_at(path, L.offset, L.rows * L.row);
  std::vector<double> out(n);
  fits_values(L, b.data(), 0, 0, n, out.data());
  return out;
}
// file order (RING) -> NESTED
std::vector<double> ring_to_nested(const std::vector<double>& ring) {
  const int64_t nside = nside_of(ring.size());
  int order = 0;
  while ((int64_t(1) << order) < nside) ++order;
  std::vector<double> nest(ring.size());
  for (size_t p = 0; p < ring.size(); ++p) nest[(size_t)ring2nest((i64)p, order)] = ring[p];
  return nest;
}
}  // namespace

std::vector<double> read_map(const std::string& path) {
  if (!is_fits(path)) return read_npy(path, nullptr);
  const Fits L = fits_layout(path);
  std::vector<double> v = fits_all(path, L);
  if (L.nested) {
    nside_of(v.size());  // a full-sky map, as a RING one must be
    return v;
  }
  return ring_to_nested(v);
}

std::vector<double> read_map_range(const std::string& path, size_t start, size_t end) {
  if (end < start) fail(path, "range end before its start");
  const size_t n = end - start;
  if (is_fits(path)) {
    const Fits L = fits_layout(path);
    const size_t total = L.repeat * L.rows;
    if (end > total) fail(path, "range " + std::to_string(start) + ".." + std::to_string(end) + " beyond " +
                                    std::to_string(total) + " pixels");
    if (!L.nested) {  // no range of RING pixels is a range of NESTED ones
      const std::vector<double> all = read_map(path);
      return std::vector<double>(all.begin() + start, all.begin() + end);
    }
    std::vector<double> out(n);
    if (!n) return out;
    const size_t r0 = start / L.repeat, r1 = (end + L.repeat - 1) / L.repeat;  // the rows covering the range
    const std::vector<unsigned char> b = read_at(path, L.offset + (uint64_t)r0 * L.row, (r1 - r0) * L.row);
    fits_values(L, b.data(), r0, start, end, out.data());
    return out;
  }
  const Npy L = npy_layout(path);
  if (end > L.count) fail(path, "range " + std::to_string(start) + ".." + std::to_string(end) + " beyond " +
                                    std::to_string(L.count) + " elements");
  const std::vector<unsigned char> b = read_at(path, L.offset + (uint64_t)start * L.size, n * L.size);
  std::vector<double> out(n);
  npy_values(L, b.data(), n, out.data());
  return out;
}

void write_npy(const std::string& path, const double* values, const std::vector<size_t>& shape) {
  size_t n = 1;
  for (size_t s : shape) n *= s;
  std::string b = npy_header(shape);
  const size_t h = b.size();
  b.resize(h + 8 * n);
  for (size_t i = 0; i < n; ++i) store_as<double>(reinterpret_cast<unsigned char*>(&b[h + 8 * i]), values[i], false);
  write_file(path, b);
}

void write_healpix_fits(const std::string& path, const double* values, size_t n, const std::string& column,
                        bool dbl) {
  std::string b = fits_headers(n, column, dbl);
  const size_t h = b.size(), w = dbl ? 8 : 4;
  b.resize(h + w * n);
  for (size_t i = 0; i < n; ++i) {
    unsigned char* q = reinterpret_cast<unsigned char*>(&b[h + w * i]);
    if (dbl) store_as<double>(q, values[i], true);
    else store_as<float>(q, (float)values[i], true);
  }
  pad_to_block(b, '\0');
  write_file(path, b);
}

void create_map(const std::string& path, size_t n, const std::string& column, bool dbl) {
  std::string head;
  size_t data;
  if (is_fits(path)) {
    head = fits_headers(n, column, dbl);
    data = ((dbl ? 8 : 4) * n + kBlock - 1) / kBlock * kBlock;
  } else {
    head = npy_header({n});
    data = 8 * n;
  }
  write_file(path, head);
  std::ofstream f(path, std::ios::binary | std::ios::in | std::ios::out);
  if (!f) fail(path, "cannot open for writing");
  if (data) {  // size the file: its last byte written
    f.seekp((std::streamoff)(head.size() + data - 1));
    f.put('\0');
    if (!f) fail(path, "cannot size the file");
  }
}

void write_piece(const std::string& path, size_t start, const double* values, size_t count, bool dbl) {
  uint64_t offset;
  size_t w;
  bool big;
  if (is_fits(path)) {
    const Fits L = fits_layout(path);
    if (L.repeat != 1 || L.width != (dbl ? 8u : 4u)) fail(path, "not a map created with this column type");
    if (start + count > L.rows) fail(path, "piece beyond the map");
    offset = L.offset;
    w = L.width;
    big = true;
  } else {
    const Npy L = npy_layout(path);
    if (L.kind != 'f' || L.size != 8 || L.big) fail(path, "not a float64 .npy map");
    if (start + count > L.count) fail(path, "piece beyond the map");
    offset = L.offset;
    w = 8;
    big = false;
  }
  std::string b(w * count, '\0');
  for (size_t i = 0; i < count; ++i) {
    unsigned char* q = reinterpret_cast<unsigned char*>(&b[w * i]);
    if (w == 8) store_as<double>(q, values[i], big);
    else store_as<float>(q, (float)values[i], big);
  }
  std::ofstream f(path, std::ios::binary | std::ios::in | std::ios::out);
  if (!f) fail(path, "cannot open for writing");
  f.seekp((std::streamoff)(offset + (uint64_t)start * w));
  if (!f.write(b.data(), (std::streamsize)b.size())) fail(path, "write failed");
}

}  // namespace mapio
}  // namespace stl
