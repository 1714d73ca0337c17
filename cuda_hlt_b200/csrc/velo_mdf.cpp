// MDF reader: the raw banks of one type (VP by default; UT and FTCluster for the global event
// cut) of the events of an LHCb MDF file, laid out as velo_run takes them. Follows
// MDF::read_events / read_event / read_banks (mdf/src/read_mdf.cpp:29-313) with the bank types
// of LHCbToGPU::bank_types (mdf/include/read_mdf.hpp:20-24), the record format of
// mdf/include/mdf_header.hpp and
// mdf/include/raw_bank.hpp, the checksum of LHCb::genChecksum (mdf/src/raw_helpers.cpp:8-21,
// 186-199) and the ROOT-style zlib blocks of Compression::unzip (mdf/src/compression.cpp).
//
// Record: a 48-byte header (three copies of the record size, checksum, compression byte,
// header byte {version:4, subheader words:4}, data type, one spare byte, a 28-byte subheader
// {trigger mask[4], run, orbit, bunch}), then the event's raw banks, zlib-compressed in
// ROOT blocks ("ZL", method 8, 3-byte compressed size, 3-byte expanded size, zlib stream)
// when the compression byte's low nibble is non-zero. A raw bank is {magic 0xCBCB u16,
// length u16 (with the 8-byte header), type u8, version u8, source id i16, body}, padded to
// 4 bytes. Per event the output holds: number of banks of the type, their byte offsets (one
// more than banks) and for each bank its source id followed by its body words.
#include <zlib.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/velo_b200.h"

namespace {

constexpr uint32_t kMdfHeaderBytes = 48;
constexpr uint32_t kChecksumStart = 16;  // the checksum covers the record from the compression byte on
constexpr uint16_t kBankMagic = 0xCBCB;
constexpr uint8_t kBankVP = 63;
constexpr uint8_t kBankODIN = 16;
constexpr uint32_t kRootBlockHeader = 9;

// one-at-a-time hash over signed chars (the reference reads the bytes through `const char*`)
uint32_t hash32_checksum(const uint8_t* p, size_t len)
{
  uint32_t h = 0;
  for (size_t i = 0; i < len; ++i) {
    h += static_cast<uint32_t>(static_cast<int32_t>(static_cast<int8_t>(p[i])));
    h += h << 10;
    h ^= h >> 6;
  }
  h += h << 3;
  h ^= h >> 11;
  h += h << 15;
  return h;
}

// Inflates the ROOT zlib blocks of src into out; false on any malformed block.
bool inflate_root_blocks(const uint8_t* src, size_t len, std::vector<uint8_t>& out)
{
  out.clear();
  size_t pos = 0;
  while (pos < len) {
    if (len - pos < kRootBlockHeader) return false;
    const uint8_t* b = src + pos;
    if (!(b[0] == 'Z' && b[1] == 'L' && b[2] == Z_DEFLATED)) return false;
    const size_t clen = b[3] | (static_cast<size_t>(b[4]) << 8) | (static_cast<size_t>(b[5]) << 16);
    const size_t xlen = b[6] | (static_cast<size_t>(b[7]) << 8) | (static_cast<size_t>(b[8]) << 16);
    if (clen > len - pos - kRootBlockHeader) return false;
    const size_t o = out.size();
    out.resize(o + xlen);
    z_stream zs;
    std::memset(&zs, 0, sizeof zs);
    zs.next_in = const_cast<Bytef*>(b + kRootBlockHeader);
    zs.avail_in = static_cast<uInt>(clen);
    zs.next_out = out.data() + o;
    zs.avail_out = static_cast<uInt>(xlen);
    if (inflateInit(&zs) != Z_OK) return false;
    const int rc = inflate(&zs, Z_FINISH);
    const size_t got = xlen - zs.avail_out;
    inflateEnd(&zs);
    if (rc != Z_STREAM_END || got != xlen) return false;
    pos += kRootBlockHeader + clen;
  }
  return true;
}

uint32_t rd32(const uint8_t* p)
{
  uint32_t v;
  std::memcpy(&v, p, 4);
  return v;
}

}  // namespace

struct VeloMdfEvents {
  std::vector<uint8_t> raw;          // events back to back, each 4-byte aligned
  std::vector<uint64_t> offsets{0};  // [n + 1]
  std::vector<uint32_t> run;         // ODIN run number per event (0 without ODIN)
  std::vector<uint64_t> event;       // ODIN event number per event (0 without ODIN)
};

extern "C" int velo_mdf_read_banks(const char* path, uint64_t first_event, uint64_t max_events, uint32_t bank_type,
                                   VeloMdfEvents** out)
{
  if (!path || !out || bank_type > 255 || bank_type == kBankODIN) return VELO_ERR_INVALID;
  *out = nullptr;
  FILE* f = std::fopen(path, "rb");
  if (!f) return VELO_ERR_INVALID;
  auto* ev = new VeloMdfEvents();
  std::vector<uint8_t> record, banks;
  std::vector<uint32_t> bank_words, bank_offsets;
  int status = 0;
  for (uint64_t index = 0; ev->run.size() < max_events; ++index) {
    uint8_t hdr[kMdfHeaderBytes];
    if (std::fread(hdr, 1, kMdfHeaderBytes, f) != kMdfHeaderBytes) break;  // end of file
    const uint32_t record_size = rd32(hdr);
    const uint32_t checksum = rd32(hdr + 12);
    const uint8_t compression = hdr[16] & 0x0F;
    if (record_size < kMdfHeaderBytes || (hdr[17] >> 4) != 3) {
      status = VELO_ERR_BAD_RAW;
      break;
    }
    record.resize(record_size);
    std::memcpy(record.data(), hdr, kMdfHeaderBytes);
    if (std::fread(record.data() + kMdfHeaderBytes, 1, record_size - kMdfHeaderBytes, f) !=
        record_size - kMdfHeaderBytes) {
      status = VELO_ERR_BAD_RAW;  // truncated record
      break;
    }
    if (index < first_event) continue;
    if (checksum && hash32_checksum(record.data() + kChecksumStart, record_size - kChecksumStart) != checksum) {
      status = VELO_ERR_BAD_RAW;
      break;
    }
    const uint8_t* body = record.data() + kMdfHeaderBytes;
    size_t body_len = record_size - kMdfHeaderBytes;
    if (compression) {
      if (!inflate_root_blocks(body, body_len, banks)) {
        status = VELO_ERR_BAD_RAW;
        break;
      }
      body = banks.data();
      body_len = banks.size();
    }
    // walk the banks: those of the type into the event, ODIN for the event identity
    bank_words.clear();
    bank_offsets.assign(1, 0u);
    uint32_t run = 0;
    uint64_t evno = 0;
    size_t pos = 0;
    while (pos + 8 <= body_len) {
      const uint8_t* b = body + pos;
      uint16_t magic, length;
      std::memcpy(&magic, b, 2);
      std::memcpy(&length, b + 2, 2);
      const uint8_t type = b[4];
      int16_t source;
      std::memcpy(&source, b + 6, 2);
      if (magic != kBankMagic || length < 8) {
        status = VELO_ERR_BAD_RAW;
        break;
      }
      const size_t total = (length + 3u) & ~3u;
      if (pos + total > body_len) {
        status = VELO_ERR_BAD_RAW;
        break;
      }
      const uint32_t nwords = (length - 8u) / 4u;
      if (type == kBankODIN && nwords >= 5) {
        run = rd32(b + 8);
        evno = (static_cast<uint64_t>(rd32(b + 8 + 3 * 4)) << 32) + rd32(b + 8 + 4 * 4);
      } else if (type == bank_type) {
        bank_words.push_back(static_cast<uint32_t>(static_cast<int32_t>(source)));
        for (uint32_t w = 0; w < nwords; ++w) bank_words.push_back(rd32(b + 8 + 4 * w));
        bank_offsets.push_back(static_cast<uint32_t>(bank_words.size() * 4));
      }
      pos += total;
    }
    if (status) break;
    const uint32_t n_banks = static_cast<uint32_t>(bank_offsets.size() - 1);
    const size_t o = ev->raw.size();
    const size_t bytes = 4 * (1 + bank_offsets.size() + bank_words.size());
    ev->raw.resize(o + bytes);
    uint8_t* dst = ev->raw.data() + o;
    std::memcpy(dst, &n_banks, 4);
    std::memcpy(dst + 4, bank_offsets.data(), 4 * bank_offsets.size());
    std::memcpy(dst + 4 + 4 * bank_offsets.size(), bank_words.data(), 4 * bank_words.size());
    ev->offsets.push_back(ev->raw.size());
    ev->run.push_back(run);
    ev->event.push_back(evno);
  }
  std::fclose(f);
  if (status) {
    delete ev;
    return status;
  }
  *out = ev;
  return 0;
}

extern "C" int velo_mdf_read(const char* path, uint64_t first_event, uint64_t max_events, VeloMdfEvents** out)
{
  return velo_mdf_read_banks(path, first_event, max_events, kBankVP, out);
}

extern "C" uint64_t velo_mdf_count(const VeloMdfEvents* e) { return e ? e->run.size() : 0; }
extern "C" uint64_t velo_mdf_raw_bytes(const VeloMdfEvents* e) { return e ? e->raw.size() : 0; }

extern "C" int velo_mdf_copy(const VeloMdfEvents* e, void* raw, uint64_t* offsets, uint32_t* run, uint64_t* event)
{
  if (!e) return VELO_ERR_INVALID;
  if (raw && !e->raw.empty()) std::memcpy(raw, e->raw.data(), e->raw.size());
  if (offsets) std::memcpy(offsets, e->offsets.data(), 8 * e->offsets.size());
  if (run && !e->run.empty()) std::memcpy(run, e->run.data(), 4 * e->run.size());
  if (event && !e->event.empty()) std::memcpy(event, e->event.data(), 8 * e->event.size());
  return 0;
}

extern "C" void velo_mdf_free(VeloMdfEvents* e) { delete e; }
