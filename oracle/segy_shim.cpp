// Test infrastructure (oracle): the four big-endian integer readers and writers of NRLib's
// libs/nrlib/iotools/fileio.cpp (WriteBinaryShort / ReadBinaryShort / WriteBinaryInt /
// ReadBinaryInt), restated here because fileio.cpp needs boost::filesystem, which this
// environment lacks.  Everything else the SegY oracle links (TextualHeader, BinaryHeader,
// TraceHeader, SegyGeometry, the IBM float writer) is the reference's own code.
#include <istream>
#include <ostream>

#include "iotools/fileio.hpp"

namespace {
template <typename T>
void put(std::ostream& s, T v, NRLib::Endianess e) {
  unsigned char b[sizeof(T)];
  for (size_t q = 0; q < sizeof(T); q++) {
    const unsigned char c = static_cast<unsigned char>((static_cast<unsigned long long>(v) >> (8 * q)) & 0xffu);
    b[e == NRLib::END_BIG_ENDIAN ? sizeof(T) - 1 - q : q] = c;
  }
  s.write(reinterpret_cast<const char*>(b), sizeof(T));
}
template <typename T>
T get(std::istream& s, NRLib::Endianess e) {
  unsigned char b[sizeof(T)] = {};
  s.read(reinterpret_cast<char*>(b), sizeof(T));
  unsigned long long v = 0;
  for (size_t q = 0; q < sizeof(T); q++) v |= static_cast<unsigned long long>(b[e == NRLib::END_BIG_ENDIAN ? sizeof(T) - 1 - q : q]) << (8 * q);
  return static_cast<T>(v);
}
}  // namespace

void NRLib::WriteBinaryShort(std::ostream& stream, short s, NRLib::Endianess e) { put<unsigned short>(stream, static_cast<unsigned short>(s), e); }
short NRLib::ReadBinaryShort(std::istream& stream, NRLib::Endianess e) { return static_cast<short>(get<unsigned short>(stream, e)); }
void NRLib::WriteBinaryInt(std::ostream& stream, int i, NRLib::Endianess e) { put<unsigned int>(stream, static_cast<unsigned int>(i), e); }
int NRLib::ReadBinaryInt(std::istream& stream, NRLib::Endianess e) { return static_cast<int>(get<unsigned int>(stream, e)); }
