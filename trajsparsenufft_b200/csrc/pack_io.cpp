// packed_header_v2 directories: writer (with the sha256 manifest the reference emits)
// and the checked reader used by plan creation.
#include "pack_io.hpp"

#include <sys/stat.h>

#include <cerrno>
#include <cstdio>
#include <fstream>
#include <sstream>

namespace tsn {

// ---- SHA-256 (FIPS 180-4) ----------------------------------------------------------------
namespace {
struct Sha256 {
  uint32_t h[8] = {0x6a09e667u, 0xbb67ae85u, 0x3c6ef372u, 0xa54ff53au,
                   0x510e527fu, 0x9b05688cu, 0x1f83d9abu, 0x5be0cd19u};
  uint8_t buf[64];
  size_t used = 0;
  uint64_t total = 0;
  static uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
  void block(const uint8_t* p) {
    static const uint32_t k[64] = {
        0x428a2f98u, 0x71374491u, 0xb5c0fbcfu, 0xe9b5dba5u, 0x3956c25bu, 0x59f111f1u, 0x923f82a4u, 0xab1c5ed5u,
        0xd807aa98u, 0x12835b01u, 0x243185beu, 0x550c7dc3u, 0x72be5d74u, 0x80deb1feu, 0x9bdc06a7u, 0xc19bf174u,
        0xe49b69c1u, 0xefbe4786u, 0x0fc19dc6u, 0x240ca1ccu, 0x2de92c6fu, 0x4a7484aau, 0x5cb0a9dcu, 0x76f988dau,
        0x983e5152u, 0xa831c66du, 0xb00327c8u, 0xbf597fc7u, 0xc6e00bf3u, 0xd5a79147u, 0x06ca6351u, 0x14292967u,
        0x27b70a85u, 0x2e1b2138u, 0x4d2c6dfcu, 0x53380d13u, 0x650a7354u, 0x766a0abbu, 0x81c2c92eu, 0x92722c85u,
        0xa2bfe8a1u, 0xa81a664bu, 0xc24b8b70u, 0xc76c51a3u, 0xd192e819u, 0xd6990624u, 0xf40e3585u, 0x106aa070u,
        0x19a4c116u, 0x1e376c08u, 0x2748774cu, 0x34b0bcb5u, 0x391c0cb3u, 0x4ed8aa4au, 0x5b9cca4fu, 0x682e6ff3u,
        0x748f82eeu, 0x78a5636fu, 0x84c87814u, 0x8cc70208u, 0x90befffau, 0xa4506cebu, 0xbef9a3f7u, 0xc67178f2u};
    uint32_t w[64];
    for (int i = 0; i < 16; ++i)
      w[i] = (uint32_t(p[4 * i]) << 24) | (uint32_t(p[4 * i + 1]) << 16) | (uint32_t(p[4 * i + 2]) << 8) | p[4 * i + 3];
    for (int i = 16; i < 64; ++i) {
      const uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
      const uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
      w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
    for (int i = 0; i < 64; ++i) {
      const uint32_t t1 = hh + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) + k[i] + w[i];
      const uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
      hh = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
  }
  void update(const uint8_t* p, size_t n) {
    total += n;
    while (n) {
      const size_t take = std::min(n, sizeof buf - used);
      std::memcpy(buf + used, p, take);
      used += take; p += take; n -= take;
      if (used == 64) { block(buf); used = 0; }
    }
  }
  std::string hex() {
    const uint64_t bits = total * 8;
    const uint8_t one = 0x80, zero = 0;
    update(&one, 1);
    while (used != 56) update(&zero, 1);
    uint8_t len[8];
    for (int i = 0; i < 8; ++i) len[i] = static_cast<uint8_t>(bits >> (56 - 8 * i));
    update(len, 8);
    char out[65];
    for (int i = 0; i < 8; ++i) std::snprintf(out + 8 * i, 9, "%08x", h[i]);
    return std::string(out, 64);
  }
};
}  // namespace

std::string sha256_hex(const void* data, size_t n) {
  Sha256 s;
  s.update(static_cast<const uint8_t*>(data), n);
  return s.hex();
}

void make_dirs(const std::string& path) {
  std::string cur;
  std::stringstream ss(path);
  std::string part;
  if (!path.empty() && path[0] == '/') cur = "/";
  while (std::getline(ss, part, '/')) {
    if (part.empty()) continue;
    cur += part + "/";
    if (mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST) fail(TSN_ERR_IO, "cannot create directory " + cur);
  }
}

FileEntry write_file(const std::string& dir, const std::string& name, const void* data, size_t bytes,
                     const std::string& dtype, std::vector<int64_t> shape) {
  const std::string path = dir + "/" + name;
  std::FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) fail(TSN_ERR_IO, "cannot open " + path);
  const size_t wrote = bytes ? std::fwrite(data, 1, bytes, f) : 0;
  if (std::fclose(f) != 0 || wrote != bytes) fail(TSN_ERR_IO, "short write " + path);
  FileEntry e;
  e.file = name;
  e.dtype = dtype;
  e.shape = std::move(shape);
  e.bytes = static_cast<int64_t>(bytes);
  e.sha256 = sha256_hex(data, bytes);
  return e;
}

void write_manifest(const std::string& dir, const std::vector<std::pair<std::string, std::string>>& fields,
                    const std::vector<FileEntry>& files) {
  std::ostringstream o;
  o << "{\n";
  for (const auto& kv : fields) o << "  \"" << kv.first << "\": " << kv.second << ",\n";
  o << "  \"files\": [\n";
  for (size_t i = 0; i < files.size(); ++i) {
    const auto& e = files[i];
    o << "    {\"bytes\": " << e.bytes << ", \"dtype\": \"" << e.dtype << "\", \"file\": \"" << e.file
      << "\", \"sha256\": \"" << e.sha256 << "\", \"shape\": [";
    for (size_t k = 0; k < e.shape.size(); ++k) o << (k ? ", " : "") << e.shape[k];
    o << "]}" << (i + 1 < files.size() ? "," : "") << "\n";
  }
  o << "  ]\n}\n";
  const std::string text = o.str();
  write_file(dir, "manifest.json", text.data(), text.size(), "json", {});
}

std::string read_file(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) fail(TSN_ERR_IO, "cannot open " + path);
  std::ostringstream ss;
  ss << in.rdbuf();
  return ss.str();
}

template <class T>
static std::vector<T> read_array(const std::string& path, size_t count) {
  const std::string bytes = read_file(path);
  if (bytes.size() != count * sizeof(T))
    fail(TSN_ERR_IO, "short or oversized array " + path + " (" + std::to_string(bytes.size()) + " bytes, expected " +
                         std::to_string(count * sizeof(T)) + ")");
  std::vector<T> v(count);
  if (count) std::memcpy(v.data(), bytes.data(), bytes.size());
  return v;
}

PackArrays read_pack_dir(const std::string& dir) {
  PackArrays p;
  p.h = parse_header(read_file(dir + "/header.bin"));
  const size_t groups = p.h.groups, tiles = p.h.tiles;
  p.group_offsets = read_array<uint32_t>(dir + "/group_offsets.bin", groups + 1);
  p.group_row_ids = read_array<int32_t>(dir + "/group_row_ids.bin", groups * kMTile);
  p.tile_col_ids = read_array<int32_t>(dir + "/tile_col_ids.bin", tiles * kKTile);
  p.tile_a_comp = read_array<uint16_t>(dir + "/tile_a_comp.bin", tiles * kMTile * (kKTile / 2));
  p.tile_pair_meta = read_array<uint32_t>(dir + "/tile_pair_meta.bin", tiles * kMTile);
  if (p.group_offsets.front() != 0 || p.group_offsets.back() != tiles)
    fail(TSN_ERR_FORMAT, "group offsets do not cover the tiles");
  for (size_t g = 0; g < groups; ++g)
    if (p.group_offsets[g] > p.group_offsets[g + 1]) fail(TSN_ERR_FORMAT, "group offsets are not monotone");
  for (int32_t c : p.tile_col_ids)
    if (c < 0 || static_cast<uint32_t>(c) >= p.h.n_cols) fail(TSN_ERR_FORMAT, "tile column id out of range");
  for (int32_t r : p.group_row_ids)
    if (r < -1 || (r >= 0 && static_cast<uint32_t>(r) >= p.h.output_size))
      fail(TSN_ERR_FORMAT, "group row id out of range");
  for (size_t i = 0; i < p.tile_pair_meta.size(); ++i) {
    // every 4-bit code must select two distinct ordered positions (p0 < p1)
    const uint32_t* pm = &p.tile_pair_meta[(i / kMTile) * kMTile];
    if (i % kMTile) continue;
    uint32_t row_meta[kMTile];
    for (int g = 0; g < 8; ++g) {
      const uint32_t a = pm[2 * g], b = pm[2 * g + 1];
      row_meta[g] = (a & 0xFFFFu) | ((b & 0xFFFFu) << 16);
      row_meta[g + 8] = (a >> 16) | (b & 0xFFFF0000u);
    }
    for (int r = 0; r < kMTile; ++r)
      for (int q = 0; q < 8; ++q) {
        const uint32_t code = (row_meta[r] >> (4 * q)) & 0xFu;
        if ((code & 3u) >= ((code >> 2) & 3u)) fail(TSN_ERR_FORMAT, "invalid 2:4 metadata code");
      }
  }
  return p;
}

}  // namespace tsn
