// Reader of snarkjs Groth16 proving keys (.zkey): the on-disk form whose point sections the
// reference's Msm::upload_bases_montgomery_256 takes as they are (src/msm.rs:190-197: "the form
// ffjavascript and snarkjs keep points in").
//
// Layout (little-endian): "zkey", version u32 (1), section count u32; then sections, each a type
// u32, a byte size u64 and the bytes. Section 1 holds the protocol id (1 = Groth16). Section 2
// (Groth16 header): n8q u32, q (n8q bytes), n8r u32, r (n8r bytes), nVars u32, nPublic u32,
// domainSize u32, then alpha1, beta1 (G1), beta2, gamma2 (G2), delta1 (G1), delta2 (G2). Point
// sections: 3 IC (nPublic + 1 G1 points), 5 A (nVars G1), 6 B1 (nVars G1), 7 B2 (nVars G2),
// 8 C (nVars - nPublic - 1 G1), 9 H (domainSize G1). A G1 point is x then y, a G2 point x.c0,
// x.c1, y.c0, y.c1, each coordinate n8q = 32 bytes in Montgomery form with R = 2^256; the point at
// infinity is all zeros. Section 4 (constraint coefficients) and 10 (contributions) are not
// needed by the MSMs and are skipped.
#pragma once
#include <cstdint>
#include <map>
#include <vector>

#include "runtime.hpp"

namespace zkg {

struct Zkey {
  uint32_t protocol = 0, n_vars = 0, n_public = 0, domain_size = 0;
  // Point sections (3, 5, 6, 7, 8, 9) as 32-bit words, copied out of the file image so that they
  // are aligned for the upload.
  std::map<uint32_t, std::vector<uint32_t>> points;
};

// Parses a file image; ZKG_EINVAL with the reason for anything malformed or not BN254 Groth16.
Zkey parse_zkey(const uint8_t* data, size_t len);
// G1 (1) or G2 (2) for a point section, 0 for any other section.
int zkey_section_group(uint32_t section);
// Points a section must hold, from the header.
size_t zkey_section_points(const Zkey& z, uint32_t section);

}  // namespace zkg

struct zkg_zkey {
  zkg::Zkey key;
};
