// Flow-field checkpoint files in the HDF5 format, read and written without the HDF5 library.
//
// The reference reads and writes its checkpoints through the HDF5 library (src/hdf5io.F90):
// write_io_tree (src/readwrite.F90:1920-1979) creates flowfield.h5 with the 3-D real(8) datasets
// ro, u1, u2, u3, p, t of Fortran shape (ia+1, ja+1, ka+1) (h5wa3d_r8_struct, hdf5io.F90:752-808),
// h5srite then adds the 1-element datasets nstep and time (h5_write1int / h5_write1rl8,
// hdf5io.F90:1015-1100, opening the file read-write), and readcheckpoint
// (src/readwrite.F90:1378-1528) reads them back, as 3-D blocks (h5ra3d_r8_struct,
// hdf5io.F90:204-256) or as 1-D "stream" arrays (h5ra3d_r8_stream, hdf5io.F90:258-348).
//
// Neither this image nor the GPU machines carry the HDF5 library, so this file implements the
// part of the published HDF5 file format (File Format Specification versions 2.0/3.0, The HDF
// Group) those files use:
//   reading: superblocks version 0-3 (a user block before it is skipped), object headers version 1
//            and 2 with continuation blocks, the root group as a symbol table (version 1 B-tree of
//            group nodes, symbol table nodes, local heap) or as compact link messages, datasets of
//            IEEE float or integer elements (either byte order) with compact or contiguous storage;
//            chunked, filtered (compressed) and densely linked data are refused (UNSUPPORTED);
//   writing: what the library writes by default for these calls: superblock version 0 with
//            8-byte addresses, the root group as a symbol table, version 1 object headers with the
//            fill value (version 1), datatype, dataspace (version 1) and layout (version 3,
//            contiguous) messages, little-endian IEEE doubles and 32-bit integers;
//   read-write: datasets added to an existing version-0 file whose root group is a symbol table
//            (the h5srite calls): the group's heap, nodes and B-tree are rewritten after the end
//            of the file and the root's symbol table message and the superblock are updated.
// All integers in the format are little-endian; addresses are relative to the superblock's base.

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/astr_b200.h"
#include "h5file.h"

namespace {

constexpr uint64_t UNDEF = ~uint64_t(0);
const uint8_t SIG[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
constexpr int LEAF_K = 4;       // symbol table node capacity 2K = 8 (the library's default)
constexpr int NODE_K = 16;      // group B-tree node capacity 2K = 32 children
constexpr int MAX_RANK = 32;

struct H5Fail {
  int code;
  std::string msg;
};
[[noreturn]] void bad(const std::string& m, int code = ASTR_ERR_ARG) { throw H5Fail{code, m}; }

uint64_t le(const uint8_t* p, int n) {
  uint64_t v = 0;
  for (int i = n - 1; i >= 0; --i) v = (v << 8) | p[i];
  return v;
}
void put(std::vector<uint8_t>& b, uint64_t v, int n) {
  for (int i = 0; i < n; ++i) b.push_back(uint8_t(v >> (8 * i)));
}
void pad8(std::vector<uint8_t>& b) {
  while (b.size() % 8) b.push_back(0);
}

struct Member {
  std::string name;
  uint64_t oh = UNDEF;            // object header address
  bool dataset = false;
  int cls = -1, esize = 0;        // datatype class (0 integer, 1 float; -1 other) and size in bytes
  bool be = false, sgn = false;
  std::vector<uint64_t> dims;     // dataspace, slowest first (the file's order)
  int layout = -1;                // 0 compact, 1 contiguous, 2 other (chunked, virtual)
  uint64_t addr = UNDEF, nbytes = 0;
  std::vector<uint8_t> compact;
  bool filtered = false;
};

struct Msg {
  int type = 0;
  int flags = 0;                  // bit 1: the data is a reference to a shared message
  uint64_t at = 0;                // absolute file offset of the message data
  std::vector<uint8_t> d;
};

}  // namespace

struct astr_h5 {
  int fd = -1;
  int mode = 0;                   // 0 read, 1 write, 2 read-write
  std::string path, err;
  uint64_t base = 0;              // absolute offset of the superblock (addresses are relative to it)
  int sbver = 0;
  uint64_t eoa = 0;               // next free relative address (write / read-write)
  uint64_t fsize = 0;             // file size when opened (bounds every metadata read)
  uint64_t root = UNDEF;
  uint64_t stab_at = UNDEF;       // absolute offset of the root symbol table message's data
  std::vector<Member> members;
  std::map<std::string, size_t> index;
  bool modified = false;
};

namespace {

thread_local std::string g_open_err;

// ---------------------------------------------------------------------------- file access
void pread_all(const astr_h5* h, uint64_t abs, void* buf, size_t n) {
  uint8_t* p = static_cast<uint8_t*>(buf);
  while (n) {
    ssize_t r = ::pread(h->fd, p, n, off_t(abs));
    if (r < 0 && errno == EINTR) continue;
    if (r <= 0) bad("read past the end of " + h->path + " (truncated or corrupt file)", ASTR_ERR_STATE);
    p += r; n -= size_t(r); abs += uint64_t(r);
  }
}
void pwrite_all(const astr_h5* h, uint64_t abs, const void* buf, size_t n) {
  const uint8_t* p = static_cast<const uint8_t*>(buf);
  while (n) {
    ssize_t r = ::pwrite(h->fd, p, n, off_t(abs));
    if (r < 0 && errno == EINTR) continue;
    if (r <= 0) bad("write to " + h->path + " failed: " + std::strerror(errno), ASTR_ERR_STATE);
    p += r; n -= size_t(r); abs += uint64_t(r);
  }
}
// Metadata (superblock, object headers, heaps, nodes) at relative address rel: it must lie inside
// the file as opened, so a corrupt size or address fails here without a large allocation.
std::vector<uint8_t> at(const astr_h5* h, uint64_t rel, size_t n) {
  if (rel == UNDEF || rel > h->fsize || n > h->fsize || h->base + rel + n > h->fsize)
    bad("metadata outside the file " + h->path + " (truncated or corrupt file)", ASTR_ERR_STATE);
  if (n > (size_t(256) << 20)) bad("metadata block larger than 256 MB in " + h->path + " (corrupt file)", ASTR_ERR_STATE);
  std::vector<uint8_t> b(n);
  if (n) pread_all(h, h->base + rel, b.data(), n);
  return b;
}

// ---------------------------------------------------------------------------- reading
void superblock(astr_h5* h) {
  struct stat st{};
  if (fstat(h->fd, &st) != 0) bad("cannot stat " + h->path, ASTR_ERR_STATE);
  uint64_t size = uint64_t(st.st_size), off = 0;
  h->fsize = size;
  uint8_t b[128] = {0};
  for (;;) {
    if (off + 8 > size) bad(h->path + " is not an HDF5 file (no signature)", ASTR_ERR_STATE);
    pread_all(h, off, b, 8);
    if (!std::memcmp(b, SIG, 8)) break;
    off = off ? 2 * off : 512;
  }
  pread_all(h, off, b, std::min<uint64_t>(128, size - off));
  h->sbver = b[8];
  if (h->sbver <= 1) {
    if (b[13] != 8 || b[14] != 8) bad("only 8-byte addresses and lengths are supported", ASTR_ERR_UNSUPPORTED);
    int q = 24 + (h->sbver == 1 ? 4 : 0);
    h->base = le(b + q, 8);
    h->eoa = le(b + q + 16, 8);
    h->root = le(b + q + 32 + 8, 8);
  } else if (h->sbver <= 3) {
    if (b[9] != 8 || b[10] != 8) bad("only 8-byte addresses and lengths are supported", ASTR_ERR_UNSUPPORTED);
    h->base = le(b + 12, 8);
    h->eoa = le(b + 28, 8);
    h->root = le(b + 36, 8);
  } else {
    bad("superblock version " + std::to_string(h->sbver), ASTR_ERR_UNSUPPORTED);
  }
  if (h->base != off) bad("superblock base address differs from its position", ASTR_ERR_UNSUPPORTED);
}

// The messages of the object header at rel, following continuation blocks.
std::vector<Msg> object_header(const astr_h5* h, uint64_t rel) {
  std::vector<Msg> out;
  std::vector<uint8_t> p = at(h, rel, 16);
  struct Chunk { uint64_t rel, size; };
  std::vector<Chunk> chunks;
  int ver, hs, flags = 0;
  uint64_t nmesgs = 0;
  if (!std::memcmp(p.data(), "OHDR", 4)) {
    if (p[4] != 2) bad("object header version", ASTR_ERR_STATE);
    ver = 2;
    flags = p[5];
    uint64_t pos = 6 + ((flags & 0x20) ? 16 : 0) + ((flags & 0x10) ? 4 : 0);
    int w = 1 << (flags & 3);
    std::vector<uint8_t> s = at(h, rel + pos, size_t(w));
    chunks.push_back({rel + pos + uint64_t(w), le(s.data(), w)});
    hs = 4 + ((flags & 0x04) ? 2 : 0);
  } else {
    if (p[0] != 1) bad("object header version", ASTR_ERR_STATE);
    ver = 1;
    nmesgs = le(p.data() + 2, 2);
    chunks.push_back({rel + 16, le(p.data() + 8, 4)});
    hs = 8;
  }
  for (size_t c = 0; c < chunks.size(); ++c) {
    if (c > 64) bad("too many object header continuation blocks", ASTR_ERR_STATE);
    uint64_t start = chunks[c].rel, size = chunks[c].size;
    if (ver == 2 && c > 0) {
      std::vector<uint8_t> s = at(h, start, 4);
      if (std::memcmp(s.data(), "OCHK", 4)) bad("object header continuation signature", ASTR_ERR_STATE);
      if (size < 8) bad("object header continuation size", ASTR_ERR_STATE);
      start += 4; size -= 8;
    }
    std::vector<uint8_t> body = at(h, start, size_t(size));
    uint64_t pos = 0;
    while (pos + uint64_t(hs) <= size) {
      Msg m;
      uint64_t ms;
      if (ver == 1) { m.type = int(le(&body[pos], 2)); ms = le(&body[pos + 2], 2); m.flags = body[pos + 4]; }
      else { m.type = body[pos]; ms = le(&body[pos + 1], 2); m.flags = body[pos + 3]; }
      if (pos + hs + ms > size) bad("object header message runs past its block", ASTR_ERR_STATE);
      m.d.assign(body.begin() + long(pos + hs), body.begin() + long(pos + hs + ms));
      m.at = h->base + start + pos + uint64_t(hs);
      if (m.type == 0x10) {
        if (ms < 16) bad("continuation message size", ASTR_ERR_STATE);
        chunks.push_back({le(m.d.data(), 8), le(m.d.data() + 8, 8)});
      }
      out.push_back(std::move(m));
      pos += uint64_t(hs) + ms;
      if (ver == 1 && out.size() == nmesgs) break;
    }
  }
  if (ver == 1 && out.size() != nmesgs) bad("object header message count", ASTR_ERR_STATE);
  return out;
}

// visits counts the nodes read so far: a corrupt tree whose children point back at its own nodes
// stops after 65536 visits instead of walking an exponential number of paths.
void btree_members(const astr_h5* h, uint64_t node, const std::vector<uint8_t>& heap,
                   std::vector<std::pair<std::string, uint64_t>>& out, int depth, int& visits) {
  if (depth > 16) bad("group B-tree too deep", ASTR_ERR_STATE);
  if (++visits > 65536 || out.size() > (size_t(1) << 20)) bad("group B-tree too large (corrupt file)", ASTR_ERR_STATE);
  std::vector<uint8_t> p = at(h, node, 24);
  if (std::memcmp(p.data(), "TREE", 4) || p[4] != 0) bad("group B-tree node", ASTR_ERR_STATE);
  int level = p[5];
  uint64_t n = le(&p[6], 2);
  std::vector<uint8_t> kc = at(h, node + 24, size_t(16 * n + 8));
  for (uint64_t i = 0; i < n; ++i) {
    uint64_t child = le(&kc[8 + 16 * i], 8);
    if (level > 0) { btree_members(h, child, heap, out, depth + 1, visits); continue; }
    std::vector<uint8_t> s = at(h, child, 8);
    if (std::memcmp(s.data(), "SNOD", 4)) bad("symbol table node", ASTR_ERR_STATE);
    uint64_t ns = le(&s[6], 2);
    std::vector<uint8_t> e = at(h, child + 8, size_t(40 * ns));
    for (uint64_t k = 0; k < ns; ++k) {
      uint64_t off = le(&e[40 * k], 8);
      if (off >= heap.size()) bad("link name outside the local heap", ASTR_ERR_STATE);
      const uint8_t* nul = static_cast<const uint8_t*>(std::memchr(&heap[off], 0, heap.size() - off));
      if (!nul) bad("unterminated link name", ASTR_ERR_STATE);
      out.emplace_back(std::string(reinterpret_cast<const char*>(&heap[off]), size_t(nul - &heap[off])),
                       le(&e[40 * k + 8], 8));
    }
  }
}

void parse_datatype(Member& m, const std::vector<uint8_t>& d) {
  if (d.size() < 8) bad("datatype message", ASTR_ERR_STATE);
  int cls = d[0] & 0x0f;
  m.esize = int(le(&d[4], 4));
  m.be = d[1] & 1;
  if (cls == 0) {
    if (d.size() < 12 || le(&d[8], 2) != 0 || le(&d[10], 2) != uint64_t(8 * m.esize)) return;
    if (m.esize != 1 && m.esize != 2 && m.esize != 4 && m.esize != 8) return;
    m.sgn = d[1] & 8;
    m.cls = 0;
  } else if (cls == 1) {
    if (d.size() < 20 || (d[1] & 0x40)) return;
    const int dbl[6] = {52, 11, 0, 52, 1023, 63}, flt[6] = {23, 8, 0, 23, 127, 31};
    const int* ieee = m.esize == 8 ? dbl : m.esize == 4 ? flt : nullptr;
    if (!ieee || d[12] != ieee[0] || d[13] != ieee[1] || d[14] != ieee[2] || d[15] != ieee[3] ||
        le(&d[16], 4) != uint64_t(ieee[4]) || d[2] != ieee[5])
      return;
    m.cls = 1;
  }
}

void parse_dataspace(Member& m, const std::vector<uint8_t>& d) {
  if (d.size() < 4) bad("dataspace message", ASTR_ERR_STATE);
  int ver = d[0], rank = d[1];
  size_t pos;
  if (ver == 1) pos = 8;
  else if (ver == 2) { pos = 4; if (d[3] == 2) { m.dims.assign(1, 0); return; } }
  else bad("dataspace version", ASTR_ERR_UNSUPPORTED);
  if (rank > MAX_RANK || d.size() < pos + 8 * size_t(rank)) bad("dataspace message", ASTR_ERR_STATE);
  m.dims.clear();
  for (int i = 0; i < rank; ++i) m.dims.push_back(le(&d[pos + 8 * size_t(i)], 8));
}

void parse_layout(Member& m, const std::vector<uint8_t>& d) {
  if (d.size() < 2) bad("layout message", ASTR_ERR_STATE);
  int ver = d[0];
  if (ver == 1 || ver == 2) {
    if (d.size() < 8) bad("layout message", ASTR_ERR_STATE);
    int nd = d[1], cls = d[2];
    size_t pos = 8;
    if (cls != 0) { if (d.size() < pos + 8) bad("layout message", ASTR_ERR_STATE); m.addr = le(&d[pos], 8); pos += 8; }
    if (d.size() < pos + 4 * size_t(nd)) bad("layout message", ASTR_ERR_STATE);
    uint64_t prod = 1;
    for (int i = 0; i < nd; ++i) prod *= le(&d[pos + 4 * size_t(i)], 4);
    pos += 4 * size_t(nd);
    if (cls == 0) {
      if (d.size() < pos + 4) bad("layout message", ASTR_ERR_STATE);
      uint64_t n = le(&d[pos], 4);
      if (d.size() < pos + 4 + n) bad("layout message", ASTR_ERR_STATE);
      m.layout = 0; m.nbytes = n;
      m.compact.assign(d.begin() + long(pos + 4), d.begin() + long(pos + 4 + n));
    } else if (cls == 1) {
      m.layout = 1; m.nbytes = prod;
    } else {
      m.layout = 2;
    }
  } else if (ver == 3 || ver == 4) {
    int cls = d[1];
    if (cls == 0) {
      if (d.size() < 4) bad("layout message", ASTR_ERR_STATE);
      uint64_t n = le(&d[2], 2);
      if (d.size() < 4 + n) bad("layout message", ASTR_ERR_STATE);
      m.layout = 0; m.nbytes = n;
      m.compact.assign(d.begin() + 4, d.begin() + long(4 + n));
    } else if (cls == 1) {
      if (d.size() < 18) bad("layout message", ASTR_ERR_STATE);
      m.layout = 1; m.addr = le(&d[2], 8); m.nbytes = le(&d[10], 8);
    } else {
      m.layout = 2;
    }
  } else {
    bad("layout version " + std::to_string(ver), ASTR_ERR_UNSUPPORTED);
  }
}

// Hard links of compact link messages (groups of version-2 object headers).
void link_members(const std::vector<Msg>& msgs, std::vector<std::pair<std::string, uint64_t>>& out) {
  for (const Msg& m : msgs) {
    const std::vector<uint8_t>& d = m.d;
    if (m.type == 0x02 && d.size() >= 10) {
      size_t pos = 2 + ((d[1] & 1) ? 8 : 0);
      if (d.size() >= pos + 8 && le(&d[pos], 8) != UNDEF) bad("dense link storage", ASTR_ERR_UNSUPPORTED);
    }
    if (m.type != 0x06 || d.size() < 3) continue;
    int fl = d[1];
    size_t pos = 2;
    int ltype = 0;
    if (fl & 0x08) ltype = d[pos++];
    if (fl & 0x04) pos += 8;
    if (fl & 0x10) pos += 1;
    int w = 1 << (fl & 3);
    if (d.size() < pos + size_t(w)) bad("link message", ASTR_ERR_STATE);
    uint64_t ln = le(&d[pos], w);
    pos += size_t(w);
    if (d.size() < pos + ln + (ltype == 0 ? 8 : 0)) bad("link message", ASTR_ERR_STATE);
    std::string name(reinterpret_cast<const char*>(d.data() + pos), size_t(ln));
    pos += ln;
    if (ltype == 0) out.emplace_back(name, le(&d[pos], 8));
  }
}

void read_structure(astr_h5* h) {
  superblock(h);
  std::vector<Msg> rm = object_header(h, h->root);
  std::vector<std::pair<std::string, uint64_t>> links;
  bool stab = false;
  for (const Msg& m : rm) {
    if (m.type != 0x11) continue;
    if (m.d.size() < 16) bad("symbol table message", ASTR_ERR_STATE);
    stab = true;
    h->stab_at = m.at;
    uint64_t heap_at = le(&m.d[8], 8);
    std::vector<uint8_t> hp = at(h, heap_at, 32);
    if (std::memcmp(hp.data(), "HEAP", 4)) bad("local heap", ASTR_ERR_STATE);
    std::vector<uint8_t> heap = at(h, le(&hp[24], 8), size_t(le(&hp[8], 8)));
    int visits = 0;
    btree_members(h, le(m.d.data(), 8), heap, links, 0, visits);
    break;
  }
  if (!stab) link_members(rm, links);
  for (auto& l : links) {
    Member mb;
    mb.name = l.first;
    mb.oh = l.second;
    bool space = false, type = false, lay = false;
    bool shared = false;
    for (const Msg& m : object_header(h, mb.oh)) {
      if ((m.type == 0x01 || m.type == 0x03) && (m.flags & 0x02)) { shared = true; space |= m.type == 0x01; type |= m.type == 0x03; }
      else if (m.type == 0x01) { parse_dataspace(mb, m.d); space = true; }
      else if (m.type == 0x03) { parse_datatype(mb, m.d); type = true; }
      else if (m.type == 0x08) { parse_layout(mb, m.d); lay = true; }
      else if (m.type == 0x0B) mb.filtered = true;
    }
    mb.dataset = space && type && lay;
    if (shared) mb.cls = -1;      // a committed (shared) datatype or dataspace: not read here
    h->index[mb.name] = h->members.size();
    h->members.push_back(std::move(mb));
  }
}

const Member& find(const astr_h5* h, const char* name) {
  if (!name) bad("null dataset name");
  auto it = h->index.find(name);
  if (it == h->index.end()) bad(std::string("no dataset '") + name + "' in " + h->path);
  const Member& m = h->members[it->second];
  if (!m.dataset) bad(std::string("'") + name + "' is not a dataset");
  return m;
}

// Elements of a dataspace, saturating (a corrupt dataspace must not wrap around).
uint64_t count(const std::vector<uint64_t>& dims) {
  uint64_t n = 1;
  for (uint64_t d : dims) {
    if (d && n > UINT64_MAX / d) return UINT64_MAX;
    n *= d;
  }
  return n;
}

template <class T>
void convert(const Member& m, const uint8_t* src, uint64_t n, T* dst) {
  for (uint64_t i = 0; i < n; ++i) {
    uint8_t b[8];
    for (int k = 0; k < m.esize; ++k) b[k] = src[i * uint64_t(m.esize) + uint64_t(m.be ? m.esize - 1 - k : k)];
    if (m.cls == 1) {
      if (m.esize == 8) { double v; std::memcpy(&v, b, 8); dst[i] = T(v); }
      else { float v; std::memcpy(&v, b, 4); dst[i] = T(v); }
    } else {
      uint64_t u = le(b, m.esize);
      if (m.sgn && m.esize < 8 && (u >> (8 * m.esize - 1))) u |= ~uint64_t(0) << (8 * m.esize);
      dst[i] = m.sgn ? T(int64_t(u)) : T(u);
    }
  }
}

// Elements [first, first + n) of the dataset, in its storage order, converted to T.
template <class T>
void read_run(const astr_h5* h, const Member& m, uint64_t first, uint64_t n, T* dst) {
  const uint64_t es = uint64_t(m.esize);
  if (m.layout == 0) {
    if ((first + n) * es > m.compact.size()) bad("compact data shorter than its dataspace", ASTR_ERR_STATE);
    convert(m, m.compact.data() + first * es, n, dst);
    return;
  }
  if (m.addr == UNDEF) {          // storage never allocated: the fill value (zero)
    std::fill(dst, dst + n, T(0));
    return;
  }
  const bool direct = sizeof(T) == size_t(m.esize) && !m.be &&
                      ((m.cls == 1 && std::is_floating_point<T>::value) || (m.cls == 0 && !std::is_floating_point<T>::value && m.sgn));
  if (direct) {
    pread_all(h, h->base + m.addr + first * es, dst, size_t(n * es));
    return;
  }
  std::vector<uint8_t> buf;
  const uint64_t piece = (uint64_t(8) << 20) / es;
  for (uint64_t done = 0; done < n; done += piece) {
    uint64_t k = std::min(piece, n - done);
    buf.resize(size_t(k * es));
    pread_all(h, h->base + m.addr + (first + done) * es, buf.data(), buf.size());
    convert(m, buf.data(), k, dst + done);
  }
}

// The block of Fortran shape fd[0..rank-1] at Fortran offsets off[] of a dataset whose file dims
// (slowest first) reverse them; mode 's': a 1-D dataset, off[0] its first element.
template <class T>
void read_block(const astr_h5* h, const char* name, int rank, const int64_t* fd, const int64_t* off, char mode, T* out) {
  const Member& m = find(h, name);
  if (m.cls < 0)
    bad(std::string("dataset '") + name + "' is not of an IEEE float or integer type (or its type is a shared message)",
        ASTR_ERR_UNSUPPORTED);
  if (m.filtered || m.layout == 2) bad(std::string("dataset '") + name + "' is chunked or filtered", ASTR_ERR_UNSUPPORTED);
  if (rank < 1 || rank > MAX_RANK || !fd) bad("bad rank or dims");
  uint64_t n = 1;
  for (int d = 0; d < rank; ++d) {
    if (fd[d] < 0 || (off && off[d] < 0)) bad("negative dims or offset");
    n *= uint64_t(fd[d]);
  }
  if (m.layout == 1 && m.addr != UNDEF && m.nbytes / uint64_t(m.esize) < count(m.dims))
    bad(std::string("dataset '") + name + "' storage shorter than its dataspace", ASTR_ERR_STATE);
  if (m.dims.empty()) {           // a scalar dataspace: one element
    if (n != 1 || (off && off[0] != 0)) bad(std::string("dataset '") + name + "' is a scalar");
    read_run(h, m, 0, 1, out);
    return;
  }
  if (mode == 's') {
    if (m.dims.size() != 1) bad(std::string("dataset '") + name + "' is not one-dimensional (stream mode)");
    uint64_t o = off ? uint64_t(off[0]) : 0;
    if (o + n > m.dims[0]) bad(std::string("dataset '") + name + "' holds fewer elements than requested");
    read_run(h, m, o, n, out);
    return;
  }
  if (mode != 'h') bad("mode must be 'h' or 's'");
  if (int(m.dims.size()) != rank) bad(std::string("dataset '") + name + "' has rank " + std::to_string(m.dims.size()));
  std::vector<uint64_t> fdim(static_cast<size_t>(rank), 0), o(static_cast<size_t>(rank), 0);
  for (int d = 0; d < rank; ++d) {
    fdim[size_t(d)] = m.dims[size_t(rank - 1 - d)];
    if (off) o[size_t(d)] = uint64_t(off[d]);
    if (o[size_t(d)] + uint64_t(fd[d]) > fdim[size_t(d)])
      bad(std::string("dataset '") + name + "' is smaller than the requested block");
  }
  if (n == 0) return;
  // the longest contiguous run: leading Fortran dims read in full, then one partial dim
  int lead = 0;
  uint64_t run = 1;
  while (lead < rank && uint64_t(fd[lead]) == fdim[size_t(lead)] && o[size_t(lead)] == 0) run *= fdim[size_t(lead++)];
  if (lead < rank) run *= uint64_t(fd[lead++]);
  std::vector<uint64_t> idx(static_cast<size_t>(rank), 0);
  for (uint64_t done = 0; done < n; done += run) {
    // storage index of the run's first element
    uint64_t lin = 0;
    for (int d = rank - 1; d >= 0; --d) lin = lin * fdim[size_t(d)] + o[size_t(d)] + (d >= lead ? idx[size_t(d)] : 0);
    read_run(h, m, lin, run, out + done);
    for (int d = lead; d < rank; ++d) {
      if (++idx[size_t(d)] < uint64_t(fd[d])) break;
      idx[size_t(d)] = 0;
    }
  }
}

// ---------------------------------------------------------------------------- writing
void message(std::vector<uint8_t>& oh, int type, int flags, std::vector<uint8_t> body) {
  pad8(body);
  put(oh, uint64_t(type), 2);
  put(oh, body.size(), 2);
  oh.push_back(uint8_t(flags));
  put(oh, 0, 3);
  oh.insert(oh.end(), body.begin(), body.end());
}
std::vector<uint8_t> object_header_v1(const std::vector<uint8_t>& msgs, int nmsgs) {
  std::vector<uint8_t> oh;
  oh.push_back(1);
  oh.push_back(0);
  put(oh, uint64_t(nmsgs), 2);
  put(oh, 1, 4);
  put(oh, msgs.size(), 4);
  put(oh, 0, 4);
  oh.insert(oh.end(), msgs.begin(), msgs.end());
  return oh;
}

uint64_t append(astr_h5* h, const void* p, uint64_t n) {
  h->eoa = (h->eoa + 7) & ~uint64_t(7);
  uint64_t a = h->eoa;
  if (n) pwrite_all(h, h->base + a, p, size_t(n));
  h->eoa += n;
  return a;
}

// Writes a dataset's object header and its data; with reserve_only, the data's storage is only
// reserved (the caller writes it). Returns the absolute file offset of the data.
uint64_t write_dataset(astr_h5* h, const char* name, int rank, const int64_t* fd, const void* data, int cls,
                       int esize, bool reserve_only = false) {
  if (h->mode == 0) bad(h->path + " is open for reading");
  if (!name || !*name || std::strchr(name, '/') || !std::strcmp(name, ".")) bad("invalid dataset name");
  if (h->index.count(name)) bad(std::string("dataset '") + name + "' already exists");
  if (rank < 1 || rank > MAX_RANK || !fd) bad("bad rank or dims");
  uint64_t n = 1;
  for (int d = 0; d < rank; ++d) {
    if (fd[d] < 0) bad("negative dims");
    n *= uint64_t(fd[d]);
  }
  if (n && !data && !reserve_only) bad("null data");
  if (h->members.size() >= size_t(2 * LEAF_K * 2 * NODE_K)) bad("too many datasets in one file", ASTR_ERR_UNSUPPORTED);
  const uint64_t nbytes = n * uint64_t(esize);
  std::vector<uint8_t> msgs, dt, sp, lay;
  // fill value, version 1: allocation late, fill if set, defined, default (zero) value
  message(msgs, 0x05, 1, {1, 2, 2, 1, 0, 0, 0, 0});
  if (cls == 1) {         // IEEE double, little-endian
    dt = {0x11, 0x20, 63, 0};
    put(dt, 8, 4);
    put(dt, 0, 2); put(dt, 64, 2);
    dt.push_back(52); dt.push_back(11); dt.push_back(0); dt.push_back(52);
    put(dt, 1023, 4);
  } else {                // 32-bit signed integer, little-endian
    dt = {0x10, 0x08, 0, 0};
    put(dt, 4, 4);
    put(dt, 0, 2); put(dt, 32, 2);
  }
  message(msgs, 0x03, 1, dt);
  sp = {1, uint8_t(rank), 0, 0, 0, 0, 0, 0};
  for (int d = rank - 1; d >= 0; --d) put(sp, uint64_t(fd[d]), 8);
  message(msgs, 0x01, 0, sp);
  const uint64_t oh_len = 16 + msgs.size() + 8 + 24;
  h->eoa = (h->eoa + 7) & ~uint64_t(7);
  const uint64_t oh_at = h->eoa;
  lay = {3, 1};
  put(lay, nbytes ? oh_at + oh_len : UNDEF, 8);
  put(lay, nbytes, 8);
  message(msgs, 0x08, 1, lay);
  std::vector<uint8_t> oh = object_header_v1(msgs, 4);
  if (oh.size() != oh_len) bad("internal: object header size", ASTR_ERR_STATE);
  append(h, oh.data(), oh.size());
  if (nbytes && h->eoa != oh_at + oh_len) bad("internal: data address", ASTR_ERR_STATE);
  if (nbytes && reserve_only) {
    h->eoa += nbytes;
  } else if (nbytes) {
    const uint8_t* p = static_cast<const uint8_t*>(data);
    for (uint64_t done = 0; done < nbytes;) {
      uint64_t k = std::min<uint64_t>(nbytes - done, uint64_t(1) << 30);
      pwrite_all(h, h->base + h->eoa, p + done, size_t(k));
      h->eoa += k;
      done += k;
    }
  }
  Member mb;
  mb.name = name;
  mb.oh = oh_at;
  mb.dataset = true;
  mb.cls = cls;
  mb.esize = esize;
  mb.sgn = cls == 0;
  for (int d = rank - 1; d >= 0; --d) mb.dims.push_back(uint64_t(fd[d]));
  mb.layout = 1;
  mb.addr = nbytes ? oh_at + oh_len : UNDEF;
  mb.nbytes = nbytes;
  h->index[mb.name] = h->members.size();
  h->members.push_back(std::move(mb));
  h->modified = true;
  return h->base + oh_at + oh_len;
}

// The root group as a symbol table (local heap, symbol table nodes, one B-tree node), written
// after the data; then the root object header (new file) or its symbol table message (read-write)
// and the superblock.
void finish(astr_h5* h) {
  std::vector<const Member*> sorted;
  for (const Member& m : h->members) sorted.push_back(&m);
  std::sort(sorted.begin(), sorted.end(),
            [](const Member* a, const Member* b) { return std::strcmp(a->name.c_str(), b->name.c_str()) < 0; });
  std::vector<uint8_t> seg(8, 0);          // offset 0: the empty name
  std::map<const Member*, uint64_t> noff;
  for (const Member* m : sorted) {
    noff[m] = seg.size();
    seg.insert(seg.end(), m->name.begin(), m->name.end());
    seg.push_back(0);
    pad8(seg);
  }
  const uint64_t free_at = seg.size();
  put(seg, 1, 8);                          // the last free block: next = 1, size 16
  put(seg, 16, 8);
  h->eoa = (h->eoa + 7) & ~uint64_t(7);
  const uint64_t heap_at = h->eoa;
  std::vector<uint8_t> heap = {'H', 'E', 'A', 'P', 0, 0, 0, 0};
  put(heap, seg.size(), 8);
  put(heap, free_at, 8);
  put(heap, heap_at + 32, 8);
  heap.insert(heap.end(), seg.begin(), seg.end());
  append(h, heap.data(), heap.size());
  std::vector<uint64_t> snods, lastkey;
  const size_t cap = 2 * LEAF_K;
  for (size_t s = 0; s < sorted.size(); s += cap) {
    size_t k = std::min(cap, sorted.size() - s);
    std::vector<uint8_t> nd = {'S', 'N', 'O', 'D', 1, 0};
    put(nd, k, 2);
    for (size_t i = 0; i < cap; ++i) {
      if (i < k) {
        put(nd, noff[sorted[s + i]], 8);
        put(nd, sorted[s + i]->oh, 8);
      } else {
        put(nd, 0, 16);
      }
      put(nd, 0, 24);                      // cache type 0, reserved, scratch
    }
    snods.push_back(append(h, nd.data(), nd.size()));
    lastkey.push_back(noff[sorted[s + k - 1]]);
  }
  std::vector<uint8_t> tree = {'T', 'R', 'E', 'E', 0, 0};
  put(tree, snods.size(), 2);
  put(tree, UNDEF, 8);
  put(tree, UNDEF, 8);
  put(tree, 0, 8);
  for (size_t i = 0; i < snods.size(); ++i) {
    put(tree, snods[i], 8);
    put(tree, lastkey[i], 8);
  }
  tree.resize(24 + (2 * NODE_K + 1) * 8 + 2 * NODE_K * 8, 0);
  const uint64_t tree_at = append(h, tree.data(), tree.size());
  std::vector<uint8_t> stab;
  put(stab, tree_at, 8);
  put(stab, heap_at, 8);
  if (h->mode == 1) {
    std::vector<uint8_t> msgs;
    message(msgs, 0x11, 1, stab);
    message(msgs, 0x00, 0, {});
    std::vector<uint8_t> oh = object_header_v1(msgs, 2);
    h->root = append(h, oh.data(), oh.size());
  } else {
    pwrite_all(h, h->stab_at, stab.data(), stab.size());
  }
  std::vector<uint8_t> sb(SIG, SIG + 8);
  const uint8_t vers[8] = {0, 0, 0, 0, 0, 8, 8, 0};
  sb.insert(sb.end(), vers, vers + 8);
  put(sb, LEAF_K, 2);
  put(sb, NODE_K, 2);
  put(sb, 0, 4);
  put(sb, h->base, 8);
  put(sb, UNDEF, 8);
  put(sb, h->base + h->eoa, 8);            // end of file: an absolute address
  put(sb, UNDEF, 8);
  put(sb, 0, 8);                           // root entry: name offset, header, cache type 1, scratch
  put(sb, h->root, 8);
  put(sb, 1, 4);
  put(sb, 0, 4);
  sb.insert(sb.end(), stab.begin(), stab.end());
  pwrite_all(h, h->base, sb.data(), sb.size());
}

// ---------------------------------------------------------------------------- C ABI
int run(astr_h5* h, const std::function<void()>& f) {
  try {
    f();
    return ASTR_OK;
  } catch (const H5Fail& e) {
    if (h) h->err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    if (h) h->err = "out of host memory";
    return ASTR_ERR_NOMEM;
  }
}
}  // namespace

extern "C" {

int astr_h5io_init(const char* filename, const char* mode, astr_h5** out) {
  if (!out || !filename || !mode) return ASTR_ERR_ARG;
  *out = nullptr;
  astr_h5* h = new (std::nothrow) astr_h5;
  if (!h) return ASTR_ERR_NOMEM;
  h->path = filename;
  int rc = run(h, [&] {
    if (!std::strcmp(mode, "read")) h->mode = 0;
    else if (!std::strcmp(mode, "write")) h->mode = 1;
    else if (!std::strcmp(mode, "rdwr")) h->mode = 2;
    else bad(std::string("mode '") + mode + "' (read, write or rdwr)");
    int fl = h->mode == 0 ? O_RDONLY : h->mode == 1 ? (O_RDWR | O_CREAT | O_TRUNC) : O_RDWR;
    h->fd = ::open(filename, fl | O_CLOEXEC, 0644);
    if (h->fd < 0) bad(std::string("cannot open ") + filename + ": " + std::strerror(errno), ASTR_ERR_STATE);
    if (h->mode == 1) {
      std::vector<uint8_t> zero(96, 0);
      pwrite_all(h, 0, zero.data(), zero.size());
      h->eoa = 96;
      h->modified = true;
      return;
    }
    read_structure(h);
    if (h->mode == 2) {
      if (h->sbver != 0 || h->stab_at == UNDEF)
        bad("adding datasets needs a version-0 superblock and a symbol-table root group", ASTR_ERR_UNSUPPORTED);
      struct stat st{};
      fstat(h->fd, &st);
      uint64_t end = std::max<uint64_t>(uint64_t(st.st_size), h->eoa);
      h->eoa = end - h->base;
    }
  });
  if (rc != ASTR_OK) {
    g_open_err = h->err;
    if (h->fd >= 0) ::close(h->fd);
    delete h;
    return rc;
  }
  *out = h;
  return ASTR_OK;
}

int astr_h5io_end(astr_h5* h) {
  if (!h) return ASTR_ERR_ARG;
  int rc = ASTR_OK;
  if (h->mode != 0 && h->modified) {
    rc = run(h, [&] { finish(h); });
    if (rc != ASTR_OK) g_open_err = h->err;
  }
  if (h->fd >= 0 && ::close(h->fd) != 0 && rc == ASTR_OK) {
    g_open_err = "close failed";
    rc = ASTR_ERR_STATE;
  }
  delete h;
  return rc;
}

const char* astr_h5_last_error(const astr_h5* h) { return h ? h->err.c_str() : g_open_err.c_str(); }

int astr_h5write_r8(astr_h5* h, const char* varname, int rank, const int64_t dims[], const double* var) {
  if (!h) return ASTR_ERR_ARG;
  return run(h, [&] { write_dataset(h, varname, rank, dims, var, 1, 8); });
}

int astr_h5write_i4(astr_h5* h, const char* varname, int rank, const int64_t dims[], const int32_t* var) {
  if (!h) return ASTR_ERR_ARG;
  return run(h, [&] { write_dataset(h, varname, rank, dims, var, 0, 4); });
}

int astr_h5read_r8(astr_h5* h, const char* varname, int rank, const int64_t dims[], const int64_t offset[],
                   char mode, double* var) {
  if (!h) return ASTR_ERR_ARG;
  return run(h, [&] {
    if (!var) bad("null output");
    read_block<double>(h, varname, rank, dims, offset, mode, var);
  });
}

int astr_h5read_i4(astr_h5* h, const char* varname, int rank, const int64_t dims[], const int64_t offset[],
                   char mode, int32_t* var) {
  if (!h) return ASTR_ERR_ARG;
  return run(h, [&] {
    if (!var) bad("null output");
    const Member& m = find(h, varname);
    if (m.cls != 0) bad(std::string("dataset '") + varname + "' is not of an integer type", ASTR_ERR_UNSUPPORTED);
    uint64_t n = 1;
    for (int d = 0; d < rank && dims; ++d) n *= uint64_t(std::max<int64_t>(dims[d], 0));
    std::vector<int64_t> tmp(static_cast<size_t>(n), 0);
    read_block<int64_t>(h, varname, rank, dims, offset, mode, tmp.data());
    for (uint64_t i = 0; i < n; ++i) {
      if (tmp[i] < INT32_MIN || tmp[i] > INT32_MAX) bad(std::string("dataset '") + varname + "' overflows int32");
      var[i] = int32_t(tmp[i]);
    }
  });
}

int astr_h5_dataset_info(astr_h5* h, const char* varname, int* rank, int64_t dims[], int* type_class, int* type_size) {
  if (!h) return ASTR_ERR_ARG;
  return run(h, [&] {
    const Member& m = find(h, varname);
    if (rank) *rank = int(m.dims.size());
    if (dims)
      for (size_t d = 0; d < m.dims.size(); ++d) dims[d] = int64_t(m.dims[m.dims.size() - 1 - d]);
    if (type_class) *type_class = m.cls;
    if (type_size) *type_size = m.esize;
  });
}

int astr_h5_count(astr_h5* h, int* n) {
  if (!h || !n) return ASTR_ERR_ARG;
  *n = int(h->members.size());
  return ASTR_OK;
}

int astr_h5_name(astr_h5* h, int i, char* name, int len) {
  if (!h || !name || len <= 0 || i < 0 || size_t(i) >= h->members.size()) return ASTR_ERR_ARG;
  const std::string& s = h->members[size_t(i)].name;
  if (s.size() + 1 > size_t(len)) return ASTR_ERR_ARG;
  std::memcpy(name, s.c_str(), s.size() + 1);
  return ASTR_OK;
}

}  // extern "C"

namespace astr {

int h5_reserve_r8(astr_h5* h, const char* varname, int rank, const int64_t dims[], int* fd, uint64_t* offset) {
  if (!h || !fd || !offset) return ASTR_ERR_ARG;
  return run(h, [&] {
    *offset = write_dataset(h, varname, rank, dims, nullptr, 1, 8, true);
    *fd = h->fd;
  });
}

int h5_locate_r8(astr_h5* h, const char* varname, int rank, const int64_t dims[], char mode, int* fd,
                 uint64_t* offset) {
  if (!h || !fd || !offset || !dims || rank < 1) return ASTR_ERR_ARG;
  const auto it = h->index.find(varname ? varname : "");
  if (it == h->index.end()) return ASTR_ERR_UNSUPPORTED;
  const Member& m = h->members[it->second];
  if (!m.dataset || m.cls != 1 || m.esize != 8 || m.be || m.filtered || m.layout != 1 || m.addr == UNDEF)
    return ASTR_ERR_UNSUPPORTED;
  uint64_t n = 1;
  for (int d = 0; d < rank; ++d) n *= uint64_t(dims[d]);
  bool match;
  if (mode == 's') {
    match = m.dims.size() == 1 && m.dims[0] == n;
  } else {
    match = int(m.dims.size()) == rank;
    for (int d = 0; match && d < rank; ++d) match = m.dims[size_t(rank - 1 - d)] == uint64_t(dims[d]);
  }
  if (!match || m.nbytes < 8 * n) return ASTR_ERR_UNSUPPORTED;
  *fd = h->fd;
  *offset = h->base + m.addr;
  return ASTR_OK;
}

}  // namespace astr
