// .zkey reader (layout in zkey.hpp). Host code only: parsing needs no GPU; the point sections
// are then uploaded through the Montgomery-2^256 path (zkg_zkey_upload in capi.cu).
#include <cstring>
#include <string>

#include "host_field.hpp"
#include "zkey.hpp"

namespace zkg {

namespace {

struct Reader {
  const uint8_t* p;
  size_t len, pos = 0;
  void need(size_t k, const char* what) const {
    if (len - pos < k) fail(ZKG_EINVAL, std::string("zkey truncated in ") + what);
  }
  uint32_t u32(const char* what) {
    need(4, what);
    uint32_t v;
    std::memcpy(&v, p + pos, 4);
    pos += 4;
    return v;
  }
  uint64_t u64(const char* what) {
    need(8, what);
    uint64_t v;
    std::memcpy(&v, p + pos, 8);
    pos += 8;
    return v;
  }
};

// The 32 little-endian bytes of a field's modulus.
void modulus_bytes(const host::Field& f, uint8_t out[32]) {
  for (int i = 0; i < 4; i++)
    for (int b = 0; b < 8; b++) out[8 * i + b] = (uint8_t)(f.p.v[i] >> (8 * b));
}

}  // namespace

int zkey_section_group(uint32_t section) {
  switch (section) {
    case 3: case 5: case 6: case 8: case 9: return ZKG_G1;
    case 7: return ZKG_G2;
    default: return 0;
  }
}

size_t zkey_section_points(const Zkey& z, uint32_t section) {
  switch (section) {
    case 3: return (size_t)z.n_public + 1;
    case 5: case 6: case 7: return z.n_vars;
    case 8: return (size_t)z.n_vars - z.n_public - 1;
    case 9: return z.domain_size;
    default: return 0;
  }
}

Zkey parse_zkey(const uint8_t* data, size_t len) {
  if (!data) fail(ZKG_EINVAL, "zkey data is NULL");
  Reader r{data, len};
  r.need(4, "magic");
  if (std::memcmp(data, "zkey", 4) != 0) fail(ZKG_EINVAL, "not a zkey file (magic is not \"zkey\")");
  r.pos = 4;
  const uint32_t version = r.u32("version");
  if (version != 1) fail(ZKG_EINVAL, "zkey version " + std::to_string(version) + " is not supported (1)");
  const uint32_t nsec = r.u32("section count");
  std::map<uint32_t, std::pair<size_t, size_t>> where;  // type -> (offset, size), first occurrence
  for (uint32_t i = 0; i < nsec; i++) {
    const uint32_t type = r.u32("section header");
    const uint64_t size = r.u64("section header");
    if (size > len - r.pos) fail(ZKG_EINVAL, "zkey section " + std::to_string(type) + " truncated");
    if (!where.count(type)) where[type] = {r.pos, (size_t)size};
    r.pos += (size_t)size;
  }
  Zkey z;
  auto section = [&](uint32_t type) -> std::pair<size_t, size_t> {
    auto it = where.find(type);
    if (it == where.end()) fail(ZKG_EINVAL, "zkey has no section " + std::to_string(type));
    return it->second;
  };
  {
    auto s = section(1);
    Reader h{data + s.first, s.second};
    z.protocol = h.u32("protocol");
    if (z.protocol != 1) fail(ZKG_EINVAL, "zkey protocol " + std::to_string(z.protocol) + " is not Groth16 (1)");
  }
  {
    auto s = section(2);
    Reader h{data + s.first, s.second};
    uint8_t want[32];
    const uint32_t n8q = h.u32("Groth16 header");
    h.need(n8q, "Groth16 header");
    modulus_bytes(host::fq(), want);
    if (n8q != 32 || std::memcmp(data + s.first + h.pos, want, 32) != 0)
      fail(ZKG_EINVAL, "zkey base field is not BN254's q");
    h.pos += n8q;
    const uint32_t n8r = h.u32("Groth16 header");
    h.need(n8r, "Groth16 header");
    modulus_bytes(host::fr(), want);
    if (n8r != 32 || std::memcmp(data + s.first + h.pos, want, 32) != 0)
      fail(ZKG_EINVAL, "zkey scalar field is not BN254's r");
    h.pos += n8r;
    z.n_vars = h.u32("Groth16 header");
    z.n_public = h.u32("Groth16 header");
    z.domain_size = h.u32("Groth16 header");
    if (z.n_vars < z.n_public + 1) fail(ZKG_EINVAL, "zkey header: nVars < nPublic + 1");
    if (z.domain_size == 0 || (z.domain_size & (z.domain_size - 1)))
      fail(ZKG_EINVAL, "zkey header: domainSize is not a power of two");
    h.need(3 * 64 + 3 * 128, "Groth16 header");  // alpha1, beta1, beta2, gamma2, delta1, delta2
  }
  for (uint32_t type : {3u, 5u, 6u, 7u, 8u, 9u}) {
    auto s = section(type);
    const size_t pts = zkey_section_points(z, type);
    const size_t bytes_per = zkey_section_group(type) == ZKG_G1 ? 64 : 128;
    if (s.second != pts * bytes_per)
      fail(ZKG_EINVAL, "zkey section " + std::to_string(type) + " holds " + std::to_string(s.second) + " bytes; " +
                           std::to_string(pts) + " points need " + std::to_string(pts * bytes_per));
    std::vector<uint32_t> w(s.second / 4);
    if (!w.empty()) std::memcpy(w.data(), data + s.first, s.second);
    // every coordinate below q (a Montgomery value x 2^256 mod q is reduced)
    const host::U256& q = host::fq().p;
    for (size_t k = 0; k < w.size(); k += 8) {
      const host::U256 v = host::from_words32(&w[k]);
      if (host::geq(v, q))
        fail(ZKG_EINVAL, "zkey section " + std::to_string(type) + ": coordinate " + std::to_string(k / 8) +
                             " is not below q");
    }
    z.points[type] = std::move(w);
  }
  return z;
}

}  // namespace zkg
