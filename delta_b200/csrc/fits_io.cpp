// FITS image layers of the reference's read_fits / write_fits
// (src/bindings.cpp:128-166 -> delta::io::read_image / write_image,
// src/io.cpp:79-178), written from the FITS standard (version 4.0): 2880-byte
// records, 80-character header cards, big-endian data, images as the primary
// HDU or IMAGE extensions. CFITSIO is not used. Host code only.
//
// Read: the primary image, or the DIFFERENCE extension when the primary holds
// no 2-D image (the compressed product layout); optional VARIANCE (as float)
// and MASK (as unsigned byte) extensions found by EXTNAME. Pixels of any
// BITPIX are converted with BSCALE / BZERO. Tile-compressed HDUs (ZIMAGE = T
// binary tables) are reported as unsupported instead of being decompressed.
// Write: a float primary image, then VARIANCE (float) and MASK (byte)
// extensions when given, as the reference lays them out.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <sys/types.h>

#include "delta_gpu.h"
#include "internal.h"

namespace dgpu {
namespace {

constexpr int64_t kRecord = 2880;
constexpr int kCard = 80;

struct File {
  std::FILE* f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace(static_cast<unsigned char>(s[a]))) ++a;
  while (b > a && std::isspace(static_cast<unsigned char>(s[b - 1]))) --b;
  return s.substr(a, b - a);
}

std::string upper(std::string s) {
  for (char& ch : s) ch = static_cast<char>(std::toupper(static_cast<unsigned char>(ch)));
  return s;
}

// One header-data unit: the keywords this reader needs, and where its data lie.
struct Hdu {
  bool primary = false;
  std::string xtension, extname;
  int bitpix = 0;
  std::vector<int64_t> naxes;
  int64_t pcount = 0, gcount = 1;
  double bscale = 1.0, bzero = 0.0;
  bool zimage = false;
  int64_t data_offset = 0, data_bytes = 0;
  int64_t pixels() const {
    if (naxes.empty()) return 0;
    int64_t n = 1;
    for (int64_t a : naxes) n *= a;
    return n;
  }
};

// Value field of a "KEYWORD = value / comment" card: the quoted string without
// its quotes (doubled quotes undone), or the token before any comment.
std::string card_value(const char* card) {
  std::string v(card + 10, card + kCard);
  size_t i = 0;
  while (i < v.size() && v[i] == ' ') ++i;
  if (i < v.size() && v[i] == '\'') {
    std::string out;
    for (size_t j = i + 1; j < v.size(); ++j) {
      if (v[j] == '\'') {
        if (j + 1 < v.size() && v[j + 1] == '\'') {
          out.push_back('\'');
          ++j;
          continue;
        }
        break;
      }
      out.push_back(v[j]);
    }
    while (!out.empty() && out.back() == ' ') out.pop_back();  // trailing blanks are not significant
    return out;
  }
  const size_t slash = v.find('/', i);
  return trim(v.substr(i, slash == std::string::npos ? std::string::npos : slash - i));
}

int64_t to_int(const std::string& v, const char* key) {
  char* end = nullptr;
  const long long x = std::strtoll(v.c_str(), &end, 10);
  if (v.empty() || end == v.c_str() || *end != '\0') fail(DGPU_ERR_RUNTIME, std::string("FITS: bad value of ") + key);
  return x;
}

double to_double(std::string v, const char* key) {
  for (char& ch : v)
    if (ch == 'D' || ch == 'd') ch = 'E';  // Fortran exponent
  char* end = nullptr;
  const double x = std::strtod(v.c_str(), &end);
  if (v.empty() || end == v.c_str() || *end != '\0') fail(DGPU_ERR_RUNTIME, std::string("FITS: bad value of ") + key);
  return x;
}

// All HDUs of the file (headers parsed, data skipped).
std::vector<Hdu> scan(std::FILE* f, const std::string& path) {
  std::vector<Hdu> hdus;
  int64_t pos = 0;
  std::vector<char> rec(kRecord);
  for (;;) {
    if (fseeko(f, static_cast<off_t>(pos), SEEK_SET) != 0) break;
    const size_t got = std::fread(rec.data(), 1, kRecord, f);
    if (got == 0) break;  // end of file: no further HDU
    if (got != static_cast<size_t>(kRecord)) fail(DGPU_ERR_RUNTIME, "FITS: truncated header in " + path);
    Hdu h;
    h.primary = hdus.empty();
    bool end = false, first = true;
    int64_t hpos = pos;
    while (!end) {
      for (int c = 0; c < kRecord / kCard && !end; ++c) {
        const char* card = rec.data() + c * kCard;
        const std::string key = trim(std::string(card, card + 8));
        if (first) {
          first = false;
          if (h.primary ? key != "SIMPLE" : key != "XTENSION")
            fail(DGPU_ERR_RUNTIME, "FITS: " + path + (h.primary ? " does not start with SIMPLE" : ": HDU without XTENSION"));
        }
        if (key == "END") {
          end = true;
          break;
        }
        if (card[8] != '=' || card[9] != ' ') continue;  // commentary card
        const std::string v = card_value(card);
        if (key == "XTENSION") h.xtension = upper(v);
        else if (key == "BITPIX") h.bitpix = static_cast<int>(to_int(v, "BITPIX"));
        else if (key == "NAXIS") h.naxes.assign(static_cast<size_t>(to_int(v, "NAXIS")), 0);
        else if (key.rfind("NAXIS", 0) == 0 && key.size() > 5) {
          const int64_t i = to_int(key.substr(5), "NAXISn");
          if (i >= 1 && i <= static_cast<int64_t>(h.naxes.size())) h.naxes[i - 1] = to_int(v, "NAXISn");
        } else if (key == "PCOUNT") h.pcount = to_int(v, "PCOUNT");
        else if (key == "GCOUNT") h.gcount = to_int(v, "GCOUNT");
        else if (key == "BSCALE") h.bscale = to_double(v, "BSCALE");
        else if (key == "BZERO") h.bzero = to_double(v, "BZERO");
        else if (key == "EXTNAME") h.extname = upper(v);
        else if (key == "ZIMAGE") h.zimage = upper(v) == "T";
      }
      hpos += kRecord;
      if (!end) {
        if (std::fread(rec.data(), 1, kRecord, f) != static_cast<size_t>(kRecord))
          fail(DGPU_ERR_RUNTIME, "FITS: header without END in " + path);
      }
    }
    const int64_t bytes_per = std::abs(h.bitpix) / 8;
    if (bytes_per != 1 && bytes_per != 2 && bytes_per != 4 && bytes_per != 8)
      fail(DGPU_ERR_RUNTIME, "FITS: unsupported BITPIX in " + path);
    // Sizes from the header are untrusted: negative axes or counts would move
    // the next HDU's offset backwards (re-parsing earlier headers forever), and
    // large ones could overflow the byte count. Both are refused, as CFITSIO does.
    if (h.pcount < 0) fail(DGPU_ERR_RUNTIME, "FITS: negative PCOUNT in " + path);
    if (h.gcount < 1) fail(DGPU_ERR_RUNTIME, "FITS: GCOUNT below 1 in " + path);
    constexpr int64_t kMaxBytes = int64_t(1) << 60;
    int64_t nax = h.naxes.empty() ? 0 : 1;
    for (int64_t a : h.naxes) {
      if (a < 0) fail(DGPU_ERR_RUNTIME, "FITS: negative NAXISn in " + path);
      if (a > 0 && nax > kMaxBytes / a) fail(DGPU_ERR_RUNTIME, "FITS: data size overflows in " + path);
      nax *= a;
    }
    if (h.pcount > kMaxBytes - nax || (h.pcount + nax) > kMaxBytes / (bytes_per * h.gcount))
      fail(DGPU_ERR_RUNTIME, "FITS: data size overflows in " + path);
    h.data_offset = hpos;
    h.data_bytes = bytes_per * h.gcount * (h.pcount + nax);
    hdus.push_back(h);
    const int64_t next = hpos + (h.data_bytes + kRecord - 1) / kRecord * kRecord;
    if (next <= pos) fail(DGPU_ERR_RUNTIME, "FITS: HDU layout does not advance in " + path);
    pos = next;
  }
  if (hdus.empty()) fail(DGPU_ERR_RUNTIME, "FITS: " + path + " holds no HDU");
  return hdus;
}

const Hdu* named(const std::vector<Hdu>& hdus, const char* name) {
  for (const Hdu& h : hdus)
    if (!h.primary && h.extname == name) return &h;
  return nullptr;
}

bool is_image(const Hdu& h) { return h.primary || h.xtension == "IMAGE"; }

void require_plain(const Hdu& h, const std::string& what) {
  if (h.zimage)
    fail(DGPU_ERR_RUNTIME, "FITS: " + what + " is a tile-compressed HDU; only uncompressed images are supported");
  if (!is_image(h)) fail(DGPU_ERR_RUNTIME, "FITS: " + what + " is not an image HDU");
}

// The image HDU that holds the data layer (delta::io::read_image's choice).
const Hdu& data_hdu(const std::vector<Hdu>& hdus, const std::string& path) {
  const Hdu& p = hdus.front();
  if (p.naxes.size() == 2) return p;
  const Hdu* d = named(hdus, "DIFFERENCE");
  if (!d)
    fail(DGPU_ERR_RUNTIME, "read_fits: " + path + ": primary is not a 2-D image (NAXIS=" +
                               std::to_string(p.naxes.size()) + ") and no DIFFERENCE extension was found");
  require_plain(*d, "the DIFFERENCE extension");
  if (d->naxes.size() != 2)
    fail(DGPU_ERR_RUNTIME, "read_fits: DIFFERENCE extension is not 2-D, got NAXIS=" + std::to_string(d->naxes.size()));
  return *d;
}

template <class T>
T load_be(const unsigned char* p) {
  unsigned char b[sizeof(T)];
  for (size_t i = 0; i < sizeof(T); ++i) b[i] = p[sizeof(T) - 1 - i];
  T v;
  std::memcpy(&v, b, sizeof(T));
  return v;
}

// Physical value (BZERO + BSCALE * stored) of element i of a raw big-endian buffer.
double physical(const Hdu& h, const unsigned char* raw, int64_t i) {
  double v = 0.0;
  switch (h.bitpix) {
    case 8: v = raw[i]; break;
    case 16: v = load_be<int16_t>(raw + 2 * i); break;
    case 32: v = load_be<int32_t>(raw + 4 * i); break;
    case 64: v = static_cast<double>(load_be<int64_t>(raw + 8 * i)); break;
    case -32: v = load_be<float>(raw + 4 * i); break;
    case -64: v = load_be<double>(raw + 8 * i); break;
    default: fail(DGPU_ERR_RUNTIME, "FITS: unsupported BITPIX");
  }
  return h.bzero + h.bscale * v;
}

// The first n pixels of h converted by `put(i, physical value / raw float)`,
// streamed in slices so a large layer never sits twice in memory.
template <class Put>
void read_pixels(std::FILE* f, const Hdu& h, int64_t n, const std::string& what, Put&& put) {
  if (h.pixels() < n) fail(DGPU_ERR_RUNTIME, "FITS: " + what + " holds fewer pixels than the data layer");
  const int64_t bp = std::abs(h.bitpix) / 8;
  constexpr int64_t kSlice = int64_t(1) << 20;  // pixels per read
  std::vector<unsigned char> buf(static_cast<size_t>(std::min(n, kSlice) * bp));
  if (fseeko(f, static_cast<off_t>(h.data_offset), SEEK_SET) != 0) fail(DGPU_ERR_RUNTIME, "FITS: seek failed");
  const bool plain_float = h.bitpix == -32 && h.bscale == 1.0 && h.bzero == 0.0;
  for (int64_t i0 = 0; i0 < n; i0 += kSlice) {
    const int64_t m = std::min(kSlice, n - i0);
    if (std::fread(buf.data(), 1, static_cast<size_t>(m * bp), f) != static_cast<size_t>(m * bp))
      fail(DGPU_ERR_RUNTIME, "FITS: truncated data in " + what);
    for (int64_t i = 0; i < m; ++i)
      put(i0 + i, plain_float ? static_cast<double>(load_be<float>(buf.data() + 4 * i)) : physical(h, buf.data(), i),
          plain_float);
  }
}

struct Writer {
  std::FILE* f;
  std::string path;
  int64_t written = 0;
  void bytes(const void* p, size_t n) {
    if (n && std::fwrite(p, 1, n, f) != n) fail(DGPU_ERR_RUNTIME, "write_fits: write failed for " + path);
    written += static_cast<int64_t>(n);
  }
  void pad(char fill) {
    const int64_t r = written % kRecord;
    if (r == 0) return;
    std::vector<char> z(static_cast<size_t>(kRecord - r), fill);
    bytes(z.data(), z.size());
  }
};

std::string card_int(const char* key, int64_t v, const char* comment) {
  char c[kCard + 1];
  std::snprintf(c, sizeof(c), "%-8s= %20lld / %-47s", key, static_cast<long long>(v), comment);
  return std::string(c, kCard);
}

std::string card_logical(const char* key, bool v, const char* comment) {
  char c[kCard + 1];
  std::snprintf(c, sizeof(c), "%-8s= %20s / %-47s", key, v ? "T" : "F", comment);
  return std::string(c, kCard);
}

std::string card_string(const char* key, const char* v, const char* comment) {
  char val[72];
  std::snprintf(val, sizeof(val), "'%-8s'", v);
  char c[kCard + 1];
  std::snprintf(c, sizeof(c), "%-8s= %-20s / %-47s", key, val, comment);
  return std::string(c, kCard);
}

std::string card_end() {
  std::string c(kCard, ' ');
  c.replace(0, 3, "END");
  return c;
}

void write_header(Writer& w, const std::vector<std::string>& cards) {
  for (const std::string& c : cards) w.bytes(c.data(), c.size());
  const std::string end = card_end();
  w.bytes(end.data(), end.size());
  w.pad(' ');
}

template <class T>
void write_be(Writer& w, const T* data, int64_t n) {
  constexpr int64_t kSlice = int64_t(1) << 20;
  std::vector<unsigned char> buf(static_cast<size_t>(std::min(n, kSlice)) * sizeof(T));
  for (int64_t i0 = 0; i0 < n; i0 += kSlice) {
    const int64_t m = std::min(kSlice, n - i0);
    for (int64_t i = 0; i < m; ++i) {
      unsigned char b[sizeof(T)];
      std::memcpy(b, data + i0 + i, sizeof(T));
      for (size_t k = 0; k < sizeof(T); ++k) buf[static_cast<size_t>(i) * sizeof(T) + k] = b[sizeof(T) - 1 - k];
    }
    w.bytes(buf.data(), static_cast<size_t>(m) * sizeof(T));
  }
  w.pad('\0');
}

std::vector<std::string> image_cards(bool primary, int bitpix, int64_t width, int64_t height) {
  std::vector<std::string> c;
  if (primary)
    c.push_back(card_logical("SIMPLE", true, "conforms to the FITS standard"));
  else
    c.push_back(card_string("XTENSION", "IMAGE", "image extension"));
  c.push_back(card_int("BITPIX", bitpix, "bits per data value"));
  c.push_back(card_int("NAXIS", 2, "number of data axes"));
  c.push_back(card_int("NAXIS1", width, "length of axis 1 (x)"));
  c.push_back(card_int("NAXIS2", height, "length of axis 2 (y)"));
  if (primary) {
    c.push_back(card_logical("EXTEND", true, "extensions may follow"));
  } else {
    c.push_back(card_int("PCOUNT", 0, "no parameter block"));
    c.push_back(card_int("GCOUNT", 1, "one data group"));
  }
  return c;
}

}  // namespace
}  // namespace dgpu

using namespace dgpu;

namespace {
template <class F>
int fits_guarded(F&& f) {
  try {
    f();
    return DGPU_OK;
  } catch (const Failure& e) {
    free_error() = e.what();
    return e.code;
  } catch (const std::exception& e) {
    free_error() = e.what();
    return DGPU_ERR_RUNTIME;
  }
}
}  // namespace

extern "C" {

int dgpu_fits_probe(const char* path, int64_t* width, int64_t* height, int* has_variance, int* has_mask) {
  return fits_guarded([&] {
    if (!path || !width || !height || !has_variance || !has_mask) fail(DGPU_ERR_INVALID, "fits_probe: missing argument");
    File file;
    file.f = std::fopen(path, "rb");
    if (!file.f) fail(DGPU_ERR_RUNTIME, std::string("read_fits: cannot open ") + path);
    const std::vector<Hdu> hdus = scan(file.f, path);
    const Hdu& d = data_hdu(hdus, path);
    *width = d.naxes[0];
    *height = d.naxes[1];
    *has_variance = named(hdus, "VARIANCE") != nullptr ? 1 : 0;
    *has_mask = named(hdus, "MASK") != nullptr ? 1 : 0;
  });
}

int dgpu_fits_read(const char* path, int64_t width, int64_t height, float* data, float* variance, uint8_t* mask) {
  return fits_guarded([&] {
    if (!path || !data) fail(DGPU_ERR_INVALID, "fits_read: missing argument");
    File file;
    file.f = std::fopen(path, "rb");
    if (!file.f) fail(DGPU_ERR_RUNTIME, std::string("read_fits: cannot open ") + path);
    const std::vector<Hdu> hdus = scan(file.f, path);
    const Hdu& d = data_hdu(hdus, path);
    // The caller's buffers hold width x height values each; a file whose data
    // layer is any other shape (changed since the probe, or a wrong caller
    // size) is refused before anything is written.
    if (d.naxes[0] != width || d.naxes[1] != height)
      fail(DGPU_ERR_INVALID, "read_fits: " + std::string(path) + " holds a " + std::to_string(d.naxes[0]) + " x " +
                                 std::to_string(d.naxes[1]) + " image, the buffers are " + std::to_string(width) +
                                 " x " + std::to_string(height));
    const int64_t n = d.naxes[0] * d.naxes[1];
    read_pixels(file.f, d, n, "the data layer",
                [&](int64_t i, double v, bool) { data[i] = static_cast<float>(v); });
    if (variance) {
      if (const Hdu* h = named(hdus, "VARIANCE")) {
        require_plain(*h, "the VARIANCE extension");
        read_pixels(file.f, *h, n, "the VARIANCE extension",
                    [&](int64_t i, double v, bool) { variance[i] = static_cast<float>(v); });
      }
    }
    if (mask) {
      if (const Hdu* h = named(hdus, "MASK")) {
        require_plain(*h, "the MASK extension");
        read_pixels(file.f, *h, n, "the MASK extension", [&](int64_t i, double v, bool) {
          // unsigned byte conversion: in range after scaling, fraction dropped
          if (!(v > -0.5 && v < 255.5)) fail(DGPU_ERR_RUNTIME, "read_fits: MASK value out of the unsigned byte range");
          mask[i] = static_cast<uint8_t>(v < 0.0 ? 0.0 : v);
        });
      }
    }
  });
}

int dgpu_fits_write(const char* path, int64_t width, int64_t height, const float* data, const float* variance,
                    const uint8_t* mask, int overwrite) {
  return fits_guarded([&] {
    if (!path || !data) fail(DGPU_ERR_INVALID, "write_fits: missing argument");
    if (width <= 0 || height <= 0) fail(DGPU_ERR_INVALID, "write_fits: image must be non-empty");
    if (!overwrite) {
      if (std::FILE* e = std::fopen(path, "rb")) {
        std::fclose(e);
        fail(DGPU_ERR_RUNTIME, std::string("write_fits: ") + path + " exists (pass overwrite=True)");
      }
    }
    File file;
    file.f = std::fopen(path, "wb");
    if (!file.f) fail(DGPU_ERR_RUNTIME, std::string("write_fits: cannot create ") + path);
    Writer w{file.f, path};
    const int64_t n = width * height;
    write_header(w, image_cards(true, -32, width, height));
    write_be(w, data, n);
    if (variance) {
      auto c = image_cards(false, -32, width, height);
      c.push_back(card_string("EXTNAME", "VARIANCE", "per-pixel variance (noise layer)"));
      write_header(w, c);
      write_be(w, variance, n);
    }
    if (mask) {
      auto c = image_cards(false, 8, width, height);
      c.push_back(card_string("EXTNAME", "MASK", "bad-pixel mask (0 = good)"));
      write_header(w, c);
      w.bytes(mask, static_cast<size_t>(n));
      w.pad('\0');
    }
    if (std::fflush(file.f) != 0) fail(DGPU_ERR_RUNTIME, std::string("write_fits: flush failed for ") + path);
  });
}

}  // extern "C"
