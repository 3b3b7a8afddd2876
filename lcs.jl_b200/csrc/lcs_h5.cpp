// lcs_h5.cpp -- restart files in the reference's HDF5 layout (no HDF5
// library: a reader and a writer of the subset these files use).
//
// The reference writes restarts with HDF5.jl (src/LCSIO/save.jl:40-167):
//   /flow/U, /flow/V, /flow/W, /flow/P          Float64, dims (nz, ny, nx)
//   /particles/<i>/counts                        Int64 (ranks,)
//   /particles/<i>/{id, x, y, z, u, v, w, diam}  Int64 / Float64 (nvalid,)
// and reads them back in src/LCSIO/load.jl:23-118 (`load_flow_fields!`, the
// particle loaders; `load_coarse_flow_fields!` of upsample.jl:1-45 for the
// `upsample` init).  A Julia array of size (nx, ny, nz) is the HDF5 dataset
// of dims (nz, ny, nx) with the same bytes, which is the ABI's host layout.
//
// Format subset (the HDF5 file format specification, version 0 superblock):
//  - written: superblock version 0 (8-byte offsets and lengths, group K 4/16),
//    groups as symbol tables (version 1 B-tree + local heap + symbol nodes),
//    version 1 object headers, datasets with a version 1 dataspace, IEEE
//    little-endian F64 or signed little-endian I64, a version 2 fill value
//    message (none defined) and a version 3 contiguous layout;
//  - read: the same, plus a user block before the superblock (base address),
//    object header continuation messages, multi-level group B-trees, version 2
//    dataspaces, compact layouts and unallocated (fill) datasets; anything
//    else fails with a message.
// Every read is bounds-checked against the file size.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/lcs_b200.h"

namespace {

thread_local std::string t_err;
int io_fail(int rc, const std::string& m) {
  t_err = m;
  return rc;
}

constexpr uint64_t kUndef = ~0ull;
constexpr int kLeafK = 4, kNodeK = 16;

// ---------------------------------------------------------------- reader
struct Reader {
  FILE* f = nullptr;
  uint64_t size = 0, base = 0;
  std::string err;
  ~Reader() {
    if (f) fclose(f);
  }
  bool open(const char* path) {
    f = fopen(path, "rb");
    if (!f) return fail(std::string("cannot open ") + path);
    fseeko(f, 0, SEEK_END);
    size = (uint64_t)ftello(f);
    static const unsigned char sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    for (uint64_t at = 0; at + 8 <= size && at <= (1ull << 30); at = at ? at * 2 : 512) {  // 0, 512, 1024, ...
      unsigned char s[8];
      if (!raw(at, s, 8)) return false;
      if (memcmp(s, sig, 8) == 0) return superblock(at);
    }
    return fail("not an HDF5 file");
  }
  bool fail(const std::string& m) {
    if (err.empty()) err = m;
    return false;
  }
  bool raw(uint64_t at, void* dst, uint64_t n) {
    if (at > size || n > size - at) return fail("read beyond the end of the file");
    if (fseeko(f, (off_t)at, SEEK_SET) != 0 || fread(dst, 1, n, f) != n) return fail("read error");
    return true;
  }
  bool rd(uint64_t addr, void* dst, uint64_t n) {  // address relative to the base
    if (addr == kUndef || addr > ~0ull - base) return fail("undefined address");
    return raw(base + addr, dst, n);
  }
  static uint64_t u(const unsigned char* p, int n) {
    uint64_t v = 0;
    for (int q = n - 1; q >= 0; q--) v = (v << 8) | p[q];
    return v;
  }
  uint64_t root_oh = kUndef;
  bool superblock(uint64_t at) {
    unsigned char b[96];
    if (!raw(at, b, 96)) return false;
    if (b[8] != 0 && b[8] != 1) return fail("superblock version " + std::to_string(b[8]) + " is not supported");
    if (b[13] != 8 || b[14] != 8) return fail("only 8-byte offsets and lengths are supported");
    const int extra = b[8] == 1 ? 4 : 0;  // version 1: indexed storage K + reserved
    unsigned char e[72];
    if (!raw(at + 24 + extra, e, 72)) return false;
    base = u(e, 8);
    // after the base address: free-space, EOF and driver addresses, then the
    // root group's symbol table entry (link name offset, object header, ...)
    root_oh = u(e + 40, 8);
    return true;
  }
  // messages of an object header (version 1, with continuation blocks)
  struct Msg {
    int type;
    std::vector<unsigned char> data;
  };
  bool messages(uint64_t oh, std::vector<Msg>* out) {
    unsigned char pre[16];
    if (!rd(oh, pre, 16)) return false;
    if (pre[0] != 1) return fail("object header version " + std::to_string(pre[0]) + " is not supported");
    const int nmsg = (int)u(pre + 2, 2);
    std::vector<std::pair<uint64_t, uint64_t>> blocks = {{oh + 16, u(pre + 8, 4)}};
    int seen = 0;
    for (size_t bi = 0; bi < blocks.size() && seen < nmsg; bi++) {
      if (blocks.size() > 4096) return fail("too many object header continuations");
      const uint64_t a0 = blocks[bi].first, len = blocks[bi].second;
      if (len > (1u << 26)) return fail("object header block too large");
      std::vector<unsigned char> blk(len);
      if (len && !rd(a0, blk.data(), len)) return false;
      uint64_t p = 0;
      while (p + 8 <= len && seen < nmsg) {
        const int type = (int)u(&blk[p], 2);
        const uint64_t sz = u(&blk[p + 2], 2);
        const int flags = blk[p + 4];
        if (p + 8 + sz > len) return fail("object header message overruns its block");
        seen++;
        if (flags & 2) return fail("shared object header messages are not supported");
        Msg m{type, std::vector<unsigned char>(blk.begin() + p + 8, blk.begin() + p + 8 + sz)};
        if (type == 0x10) {  // continuation: address, length
          if (sz < 16) return fail("short continuation message");
          blocks.push_back({u(m.data.data(), 8), u(m.data.data() + 8, 8)});
        } else {
          out->push_back(std::move(m));
        }
        p += 8 + sz;
      }
    }
    return true;
  }
  // children of a symbol-table group: name -> object header address
  bool children(uint64_t oh, std::map<std::string, uint64_t>* out) {
    std::vector<Msg> ms;
    if (!messages(oh, &ms)) return false;
    for (auto& m : ms)
      if (m.type == 0x11 && m.data.size() >= 16) {
        const uint64_t bt = u(m.data.data(), 8), heap = u(m.data.data() + 8, 8);
        unsigned char hh[32];
        if (!rd(heap, hh, 32)) return false;
        if (memcmp(hh, "HEAP", 4) != 0) return fail("bad local heap signature");
        const uint64_t hsize = u(hh + 8, 8), haddr = u(hh + 24, 8);
        if (hsize > (1u << 26)) return fail("local heap too large");
        std::vector<char> names(hsize + 1, 0);
        if (hsize && !rd(haddr, names.data(), hsize)) return false;
        btree_nodes = 0;
        return btree(bt, names, out, 0);
      }
    return fail("not a group (no symbol table message)");
  }
  int btree_nodes = 0;  // nodes visited in one group's B-tree (a malformed tree may loop)
  bool btree(uint64_t at, const std::vector<char>& names, std::map<std::string, uint64_t>* out, int depth) {
    if (depth > 16) return fail("group B-tree too deep");
    if (++btree_nodes > (1 << 16)) return fail("group B-tree too large");
    unsigned char hd[24];
    if (!rd(at, hd, 24)) return false;
    if (memcmp(hd, "TREE", 4) != 0) return fail("bad B-tree signature");
    if (hd[4] != 0) return fail("not a group B-tree");
    const int level = hd[5], used = (int)u(hd + 6, 2);
    std::vector<unsigned char> kc((size_t)used * 16 + 8);
    if (!rd(at + 24, kc.data(), kc.size())) return false;
    for (int q = 0; q < used; q++) {
      const uint64_t child = u(&kc[8 + (size_t)q * 16], 8);
      if (level > 0) {
        if (!btree(child, names, out, depth + 1)) return false;
        continue;
      }
      unsigned char sh[8];
      if (!rd(child, sh, 8)) return false;
      if (memcmp(sh, "SNOD", 4) != 0) return fail("bad symbol node signature");
      const int ns = (int)u(sh + 6, 2);
      std::vector<unsigned char> ents((size_t)ns * 40);
      if (ns && !rd(child + 8, ents.data(), ents.size())) return false;
      for (int e = 0; e < ns; e++) {
        const uint64_t no = u(&ents[(size_t)e * 40], 8), ohad = u(&ents[(size_t)e * 40 + 8], 8);
        if (no >= names.size()) return fail("symbol name outside the local heap");
        (*out)[std::string(&names[no])] = ohad;
      }
    }
    return true;
  }
  bool find(const std::string& path, uint64_t* oh) {
    uint64_t cur = root_oh;
    size_t p = 0;
    while (p < path.size()) {
      while (p < path.size() && path[p] == '/') p++;
      if (p >= path.size()) break;
      const size_t q = path.find('/', p);
      const std::string part = path.substr(p, q == std::string::npos ? std::string::npos : q - p);
      std::map<std::string, uint64_t> ch;
      if (!children(cur, &ch)) return false;
      auto it = ch.find(part);
      if (it == ch.end()) return fail("no object '" + part + "' in " + path);
      cur = it->second;
      p = q == std::string::npos ? path.size() : q;
    }
    *oh = cur;
    return true;
  }
  // a dataset's dims and element kind ('f' F64, 'i' I64), data read into dst
  // (when given, sized to the element count)
  bool dataset(const std::string& path, std::vector<uint64_t>* dims, char* kind, void* dst, uint64_t dst_bytes) {
    uint64_t oh;
    if (!find(path, &oh)) return false;
    return dataset_at(oh, path, dims, kind, dst, dst_bytes);
  }
  bool dataset_at(uint64_t oh, const std::string& path, std::vector<uint64_t>* dims, char* kind, void* dst,
                  uint64_t dst_bytes) {
    std::vector<Msg> ms;
    if (!messages(oh, &ms)) return false;
    bool have_space = false, have_type = false, have_layout = false;
    int lclass = -1;
    uint64_t addr = kUndef, bytes = 0;
    std::vector<unsigned char> compact;
    dims->clear();
    for (auto& m : ms) {
      const unsigned char* d = m.data.data();
      const size_t n = m.data.size();
      if (m.type == 0x01) {  // dataspace
        if (n < 8) return fail("short dataspace message");
        const int ver = d[0], rank = d[1];
        const size_t off = ver == 1 ? 8 : 4;
        if (ver == 2 && d[3] == 2) return fail(path + ": null dataspace");
        if (off + (size_t)rank * 8 > n) return fail("short dataspace message");
        for (int r = 0; r < rank; r++) dims->push_back(u(d + off + (size_t)r * 8, 8));
        have_space = true;
      } else if (m.type == 0x03) {  // datatype
        if (n < 8) return fail("short datatype message");
        const int cls = d[0] & 15;
        const uint64_t sz = u(d + 4, 4);
        if (sz != 8) return fail(path + ": only 8-byte elements are supported");
        if (d[1] & 1) return fail(path + ": big-endian data is not supported");
        if (cls == 1) *kind = 'f';
        else if (cls == 0) *kind = 'i';
        else return fail(path + ": datatype class " + std::to_string(cls) + " is not supported");
        have_type = true;
      } else if (m.type == 0x08 && n >= 8 && (d[0] == 1 || d[0] == 2)) {  // layout, versions 1-2
        lclass = d[2];
        if (lclass == 1) {
          if (n < 16) return fail("short layout message");
          addr = u(d + 8, 8);
          bytes = ~0ull;  // the extent follows from the dataspace
        } else {
          return fail(path + ": only contiguous version 1-2 layouts are supported");
        }
        have_layout = true;
      } else if (m.type == 0x08) {  // layout, version 3
        if (n < 2 || d[0] != 3) return fail(path + ": layout message version " + std::to_string(d[0]) + " is not supported");
        lclass = d[1];
        if (lclass == 1) {
          if (n < 18) return fail("short layout message");
          addr = u(d + 2, 8);
          bytes = u(d + 10, 8);
        } else if (lclass == 0) {
          if (n < 4) return fail("short layout message");
          const uint64_t cs = u(d + 2, 2);
          if (4 + cs > n) return fail("short compact layout");
          compact.assign(d + 4, d + 4 + cs);
        } else {
          return fail(path + ": chunked datasets are not supported");
        }
        have_layout = true;
      }
    }
    if (!have_space || !have_type || !have_layout) return fail(path + ": not a dataset");
    uint64_t count = 1;
    for (uint64_t v : *dims) count *= v;
    if (!dst) return true;
    if (count * 8 != dst_bytes) return fail(path + ": size mismatch (" + std::to_string(count) + " elements)");
    if (lclass == 0) {
      if (compact.size() < dst_bytes) return fail(path + ": short compact data");
      memcpy(dst, compact.data(), dst_bytes);
      return true;
    }
    if (addr == kUndef) {  // never written: the (undefined, zero) fill value
      memset(dst, 0, dst_bytes);
      return true;
    }
    if (bytes < dst_bytes) return fail(path + ": short contiguous data");
    return rd(addr, dst, dst_bytes);
  }
  // Every group and dataset under the group at `oh` (path `prefix`), with the
  // datasets' data: what a rewrite of the file keeps.
  struct Item {
    std::string path;  // "a/b/c"
    bool group = false;
    char kind = 'f';
    std::vector<uint64_t> dims;
    std::vector<unsigned char> data;
  };
  bool walk(uint64_t oh, const std::string& prefix, std::vector<Item>* out, int depth) {
    if (depth > 32) return fail("groups nested too deeply");
    std::map<std::string, uint64_t> ch;
    if (!children(oh, &ch)) return false;
    for (auto& kv : ch) {
      Item it;
      it.path = prefix.empty() ? kv.first : prefix + "/" + kv.first;
      std::vector<Msg> ms;
      if (!messages(kv.second, &ms)) return false;
      bool group = false;
      for (auto& m : ms) group = group || m.type == 0x11;
      if (group) {
        it.group = true;
        out->push_back(it);
        if (!walk(kv.second, it.path, out, depth + 1)) return false;
        continue;
      }
      if (!dataset_at(kv.second, it.path, &it.dims, &it.kind, nullptr, 0)) return false;
      uint64_t count = 1;
      for (uint64_t v : it.dims) {
        if (v && count > (1ull << 40) / v) return fail(it.path + ": dataset too large to rewrite");
        count *= v;
      }
      it.data.resize(count * 8);
      if (!dataset_at(kv.second, it.path, &it.dims, &it.kind, it.data.data(), count * 8)) return false;
      out->push_back(std::move(it));
    }
    return true;
  }
};

// ---------------------------------------------------------------- writer
struct WNode {
  std::string name;
  bool group = false;
  // dataset
  char kind = 'f';
  std::vector<uint64_t> dims;
  const void* data = nullptr;
  uint64_t bytes = 0;
  // group
  std::vector<std::unique_ptr<WNode>> kids;
  // layout
  uint64_t oh = 0, heap = 0, heap_data = 0, heap_size = 0, btree = 0, data_addr = 0;
  std::vector<uint64_t> snods;
  std::vector<uint64_t> leaves;    // leaf-level B-tree nodes under a level-1 root (groups of > 256 children)
  std::vector<uint64_t> name_off;  // heap offsets of the sorted children's names
  WNode* child(const std::string& n) {
    for (auto& k : kids)
      if (k->name == n) return k.get();
    kids.emplace_back(new WNode);
    kids.back()->name = n;
    return kids.back().get();
  }
};

struct Writer {
  WNode root;
  Writer() { root.group = true; }
  WNode* group(const std::string& path) {
    WNode* cur = &root;
    size_t p = 0;
    while (p < path.size()) {
      const size_t q = path.find('/', p);
      cur = cur->child(path.substr(p, q == std::string::npos ? std::string::npos : q - p));
      cur->group = true;
      if (q == std::string::npos) break;
      p = q + 1;
    }
    return cur;
  }
  void dataset(const std::string& gpath, const std::string& name, char kind, std::vector<uint64_t> dims,
               const void* data) {
    WNode* g = gpath.empty() ? &root : group(gpath);
    WNode* d = g->child(name);
    d->group = false;
    d->kind = kind;
    d->dims = std::move(dims);
    d->data = data;
    uint64_t c = 1;
    for (uint64_t v : d->dims) c *= v;
    d->bytes = c * 8;
  }

  static uint64_t pad8(uint64_t v) { return (v + 7) & ~7ull; }
  static size_t oh_group_size() { return 16 + 8 + 16; }
  static size_t ds_msgs_size(const WNode& d) {
    return (8 + pad8(8 + 8 * d.dims.size())) + (8 + (d.kind == 'f' ? 24 : 16)) + (8 + 8) + (8 + 24);
  }
  static constexpr uint64_t kBtreeSize = 24 + (2 * kNodeK + 1) * 8 + 2 * kNodeK * 8;
  static constexpr uint64_t kSnodSize = 8 + 2 * kLeafK * 40;

  uint64_t at = 96;  // after the superblock
  bool too_many = false;  // a group beyond 2 kNodeK x 2 kNodeK x 2 kLeafK children
  void sort_kids(WNode& g) {
    std::sort(g.kids.begin(), g.kids.end(), [](const std::unique_ptr<WNode>& a, const std::unique_ptr<WNode>& b) {
      return strcmp(a->name.c_str(), b->name.c_str()) < 0;
    });
  }
  void layout_meta(WNode& n) {
    if (n.group) {
      sort_kids(n);
      n.oh = at;
      at += oh_group_size();
      n.heap_size = 8;  // offset 0: the empty name
      n.name_off.clear();
      for (auto& k : n.kids) {
        n.name_off.push_back(n.heap_size);
        n.heap_size += pad8(k->name.size() + 1);
      }
      n.heap = at;
      at += 32;
      n.heap_data = at;
      at += n.heap_size;
      n.btree = at;
      at += kBtreeSize;
      const size_t nsn = (n.kids.size() + 2 * kLeafK - 1) / (2 * kLeafK);
      // one leaf-level node holds 2 kNodeK symbol nodes; above that a level-1
      // root indexes up to 2 kNodeK leaf nodes
      const size_t nleaf = (std::max<size_t>(nsn, 1) + 2 * kNodeK - 1) / (2 * kNodeK);
      if (nleaf > (size_t)(2 * kNodeK)) too_many = true;
      n.leaves.clear();
      if (nleaf > 1)
        for (size_t q = 0; q < nleaf; q++) {
          n.leaves.push_back(at);
          at += kBtreeSize;
        }
      n.snods.clear();
      for (size_t q = 0; q < std::max<size_t>(nsn, 1); q++) {
        n.snods.push_back(at);
        at += kSnodSize;
      }
      for (auto& k : n.kids) layout_meta(*k);
    } else {
      n.oh = at;
      at += 16 + ds_msgs_size(n);
    }
  }
  void layout_data(WNode& n) {
    if (n.group) {
      for (auto& k : n.kids) layout_data(*k);
    } else {
      at = pad8(at);
      n.data_addr = at;
      at += n.bytes;
    }
  }
  // little-endian field writers
  static void put(std::vector<unsigned char>& b, uint64_t v, int n) {
    for (int q = 0; q < n; q++) b.push_back((unsigned char)(v >> (8 * q)));
  }
  static void msg(std::vector<unsigned char>& b, int type, const std::vector<unsigned char>& data) {
    put(b, type, 2);
    put(b, data.size(), 2);
    put(b, 0, 4);
    b.insert(b.end(), data.begin(), data.end());
  }
  static void oh_prefix(std::vector<unsigned char>& b, int nmsg, uint64_t size) {
    put(b, 1, 1);
    put(b, 0, 1);
    put(b, nmsg, 2);
    put(b, 1, 4);
    put(b, size, 4);
    put(b, 0, 4);  // alignment of the messages to 8 bytes
  }
  bool emit(FILE* f, uint64_t addr, const std::vector<unsigned char>& b) {
    return fseeko(f, (off_t)addr, SEEK_SET) == 0 && fwrite(b.data(), 1, b.size(), f) == b.size();
  }
  static void entry(std::vector<unsigned char>& b, uint64_t name_off, const WNode& k) {
    put(b, name_off, 8);
    put(b, k.oh, 8);
    put(b, k.group ? 1 : 0, 4);
    put(b, 0, 4);
    put(b, k.group ? k.btree : 0, 8);
    put(b, k.group ? k.heap : 0, 8);
  }
  bool write_meta(FILE* f, const WNode& n) {
    std::vector<unsigned char> b;
    if (n.group) {
      std::vector<unsigned char> st;
      put(st, n.btree, 8);
      put(st, n.heap, 8);
      oh_prefix(b, 1, 8 + 16);
      msg(b, 0x11, st);
      if (!emit(f, n.oh, b)) return false;
      b.clear();
      b.insert(b.end(), {'H', 'E', 'A', 'P'});
      put(b, 0, 4);
      put(b, n.heap_size, 8);
      put(b, 1, 8);  // no free block (the HDF5 library's end-of-free-list offset)
      put(b, n.heap_data, 8);
      if (!emit(f, n.heap, b)) return false;
      b.assign(n.heap_size, 0);
      for (size_t q = 0; q < n.kids.size(); q++) memcpy(&b[n.name_off[q]], n.kids[q]->name.c_str(), n.kids[q]->name.size());
      if (!emit(f, n.heap_data, b)) return false;
      // B-tree over the symbol nodes: key i = the last name in child i-1
      // (key 0 = the last name before the node's first child, "" at the
      // start), child i holds the names in (key i, key i+1]
      const size_t per_leaf = 2 * kNodeK, nsn = n.snods.size();
      auto last_name = [&](size_t snod_end) -> uint64_t {  // the last name in symbol nodes [0, snod_end)
        const size_t last = std::min(n.kids.size(), snod_end * 2 * kLeafK);
        return last ? n.name_off[last - 1] : 0;
      };
      auto node = [&](int level, size_t c0, size_t c1, uint64_t left, uint64_t right, uint64_t key0,
                      const std::vector<uint64_t>& child, const std::vector<uint64_t>& key) {
        b.clear();
        b.insert(b.end(), {'T', 'R', 'E', 'E'});
        put(b, 0, 1);
        put(b, level, 1);
        put(b, c1 - c0, 2);
        put(b, left, 8);
        put(b, right, 8);
        put(b, key0, 8);
        for (size_t q = c0; q < c1; q++) {
          put(b, child[q], 8);
          put(b, key[q], 8);
        }
        b.resize(kBtreeSize, 0);
      };
      std::vector<uint64_t> snod_key(nsn);
      for (size_t q = 0; q < nsn; q++) snod_key[q] = last_name(q + 1);
      if (n.leaves.empty()) {
        node(0, 0, nsn, kUndef, kUndef, 0, n.snods, snod_key);
        if (!emit(f, n.btree, b)) return false;
      } else {
        const size_t nleaf = n.leaves.size();
        std::vector<uint64_t> leaf_key(nleaf);
        for (size_t l = 0; l < nleaf; l++) {
          const size_t s0 = l * per_leaf, s1 = std::min(nsn, s0 + per_leaf);
          leaf_key[l] = last_name(s1);
          node(0, s0, s1, l ? n.leaves[l - 1] : kUndef, l + 1 < nleaf ? n.leaves[l + 1] : kUndef,
               s0 ? last_name(s0) : 0, n.snods, snod_key);
          if (!emit(f, n.leaves[l], b)) return false;
        }
        node(1, 0, nleaf, kUndef, kUndef, 0, n.leaves, leaf_key);
        if (!emit(f, n.btree, b)) return false;
      }
      for (size_t q = 0; q < n.snods.size(); q++) {
        b.clear();
        b.insert(b.end(), {'S', 'N', 'O', 'D'});
        put(b, 1, 1);
        put(b, 0, 1);
        const size_t k0 = q * 2 * kLeafK, k1 = std::min(n.kids.size(), k0 + 2 * kLeafK);
        put(b, k1 - k0, 2);
        for (size_t k = k0; k < k1; k++) entry(b, n.name_off[k], *n.kids[k]);
        b.resize(kSnodSize, 0);
        if (!emit(f, n.snods[q], b)) return false;
      }
      for (auto& k : n.kids)
        if (!write_meta(f, *k)) return false;
      return true;
    }
    std::vector<unsigned char> sp, ty, fv, ly;
    put(sp, 1, 1);
    put(sp, n.dims.size(), 1);
    put(sp, 0, 1);
    put(sp, 0, 5);
    for (uint64_t d : n.dims) put(sp, d, 8);
    sp.resize(pad8(sp.size()), 0);
    if (n.kind == 'f') {  // IEEE F64 little-endian
      put(ty, 0x11, 1);   // version 1, class 1 (floating point)
      put(ty, 0x20, 1);   // little-endian, implied mantissa msb
      put(ty, 63, 1);     // sign bit
      put(ty, 0, 1);
      put(ty, 8, 4);
      put(ty, 0, 2);
      put(ty, 64, 2);
      put(ty, 52, 1);
      put(ty, 11, 1);
      put(ty, 0, 1);
      put(ty, 52, 1);
      put(ty, 1023, 4);
      ty.resize(24, 0);
    } else {              // signed I64 little-endian
      put(ty, 0x10, 1);   // version 1, class 0 (fixed point)
      put(ty, 0x08, 1);   // little-endian, signed
      put(ty, 0, 2);
      put(ty, 8, 4);
      put(ty, 0, 2);
      put(ty, 64, 2);
      ty.resize(16, 0);
    }
    put(fv, 2, 1);  // fill value message version 2: allocated late, written if set, none defined
    put(fv, 2, 1);
    put(fv, 2, 1);
    put(fv, 0, 1);
    fv.resize(8, 0);
    put(ly, 3, 1);  // layout version 3, contiguous
    put(ly, 1, 1);
    put(ly, n.data_addr, 8);
    put(ly, n.bytes, 8);
    ly.resize(24, 0);
    oh_prefix(b, 4, ds_msgs_size(n));
    msg(b, 0x01, sp);
    msg(b, 0x03, ty);
    msg(b, 0x05, fv);
    msg(b, 0x08, ly);
    return emit(f, n.oh, b);
  }
  bool write_data(FILE* f, const WNode& n) {
    if (n.group) {
      for (auto& k : n.kids)
        if (!write_data(f, *k)) return false;
      return true;
    }
    if (fseeko(f, (off_t)n.data_addr, SEEK_SET) != 0) return false;
    return n.bytes == 0 || fwrite(n.data, 1, n.bytes, f) == n.bytes;
  }
  int write(const char* path) {
    at = 96;
    too_many = false;
    layout_meta(root);
    if (too_many)
      return io_fail(LCS_EINVAL, "a group holds more than " + std::to_string(8 * kNodeK * kNodeK * kLeafK) + " entries");
    layout_data(root);
    const uint64_t eof = at;
    FILE* f = fopen(path, "wb");
    if (!f) return io_fail(LCS_EINVAL, std::string("cannot create ") + path);
    std::vector<unsigned char> sb = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n', 0, 0, 0, 0, 0, 8, 8, 0};
    put(sb, kLeafK, 2);
    put(sb, kNodeK, 2);
    put(sb, 0, 4);
    put(sb, 0, 8);       // base address
    put(sb, kUndef, 8);  // free-space info
    put(sb, eof, 8);
    put(sb, kUndef, 8);  // driver information
    entry(sb, 0, root);
    bool ok = emit(f, 0, sb) && write_meta(f, root) && write_data(f, root);
    ok = (fclose(f) == 0) && ok;
    return ok ? LCS_OK : io_fail(LCS_EINVAL, std::string("write error on ") + path);
  }
};

const char* kFlow[4] = {"U", "V", "W", "P"};

int handle_rc(lcs_handle* h, int rc) {
  if (rc != LCS_OK) {
    const char* m = lcs_last_error(h);
    t_err = m ? m : "call failed";
  }
  return rc;
}

}  // namespace

extern "C" {

const char* lcs_io_last_error(void) { return t_err.c_str(); }

int lcs_restart_save(lcs_handle* h, const char* path) {
  if (!h || !path) return io_fail(LCS_EINVAL, "null argument");
  lcs_config c;
  if (lcs_get_config(h, &c) != LCS_OK) return io_fail(LCS_EINVAL, "bad handle");
  const lcs_config* cfg = &c;
  const int64_t nx = cfg->dims[0], ny = cfg->dims[1], nz = cfg->dims[2], n3 = nx * ny * nz;
  std::vector<std::vector<double>> flow(4, std::vector<double>((size_t)n3));
  int rc = lcs_download_flow(h, flow[0].data(), flow[1].data(), flow[2].data(), flow[3].data());
  if (rc != LCS_OK) return handle_rc(h, rc);
  Writer w;
  for (int q = 0; q < 4; q++) w.dataset("flow", kFlow[q], 'f', {(uint64_t)nz, (uint64_t)ny, (uint64_t)nx}, flow[q].data());
  const int ns = cfg->mode == LCS_MODE_FLOW_PARTICLE ? cfg->n_species : 0;
  std::vector<std::vector<int64_t>> ids(ns), counts(ns);
  std::vector<std::vector<std::vector<double>>> pr(ns);
  static const char* kProp[7] = {"diam", "x", "y", "z", "u", "v", "w"};
  for (int s = 0; s < ns; s++) {
    const int64_t n = cfg->species[s].nvalid;
    ids[s].resize((size_t)n);
    counts[s] = {n};
    pr[s].assign(7, std::vector<double>((size_t)n));
    rc = lcs_download_particles(h, s, ids[s].data(), pr[s][0].data(), pr[s][1].data(), pr[s][2].data(),
                                pr[s][3].data(), pr[s][4].data(), pr[s][5].data(), pr[s][6].data());
    if (rc != LCS_OK) return handle_rc(h, rc);
    const std::string g = "particles/" + std::to_string(s + 1);
    w.dataset(g, "counts", 'i', {1}, counts[s].data());
    w.dataset(g, "id", 'i', {(uint64_t)n}, ids[s].data());
    for (int q = 0; q < 7; q++) w.dataset(g, kProp[q], 'f', {(uint64_t)n}, pr[s][q].data());
  }
  return w.write(path);
}

static int load_flow(lcs_handle* h, Reader& r, int64_t nx, int64_t ny, int64_t nz, bool coarse) {
  const int64_t n3 = nx * ny * nz;
  std::vector<std::vector<double>> flow(4, std::vector<double>((size_t)n3));
  for (int q = 0; q < 4; q++) {
    std::vector<uint64_t> dims;
    char kind = 0;
    if (!r.dataset(std::string("flow/") + kFlow[q], &dims, &kind, nullptr, 0)) return io_fail(LCS_EINVAL, r.err);
    if (dims.size() != 3 || dims[0] != (uint64_t)nz || dims[1] != (uint64_t)ny || dims[2] != (uint64_t)nx || kind != 'f')
      return io_fail(LCS_EINVAL, std::string("flow/") + kFlow[q] + ": expected Float64 (" + std::to_string(nz) + ", " +
                                     std::to_string(ny) + ", " + std::to_string(nx) + ")");
    if (!r.dataset(std::string("flow/") + kFlow[q], &dims, &kind, flow[q].data(), (uint64_t)n3 * 8))
      return io_fail(LCS_EINVAL, r.err);
  }
  const int rc = coarse ? lcs_upload_flow_coarse(h, flow[0].data(), flow[1].data(), flow[2].data(), flow[3].data())
                        : lcs_upload_flow(h, flow[0].data(), flow[1].data(), flow[2].data(), flow[3].data());
  return handle_rc(h, rc);
}

int lcs_restart_load(lcs_handle* h, const char* path) {
  if (!h || !path) return io_fail(LCS_EINVAL, "null argument");
  lcs_config c;
  if (lcs_get_config(h, &c) != LCS_OK) return io_fail(LCS_EINVAL, "bad handle");
  const lcs_config* cfg = &c;
  Reader r;
  if (!r.open(path)) return io_fail(LCS_EINVAL, r.err);
  int rc = load_flow(h, r, cfg->dims[0], cfg->dims[1], cfg->dims[2], false);
  if (rc != LCS_OK) return rc;
  const int ns = cfg->mode == LCS_MODE_FLOW_PARTICLE ? cfg->n_species : 0;
  static const char* kProp[7] = {"diam", "x", "y", "z", "u", "v", "w"};
  for (int s = 0; s < ns; s++) {
    const int64_t n = cfg->species[s].nvalid;
    const std::string g = "particles/" + std::to_string(s + 1) + "/";
    std::vector<uint64_t> dims;
    char kind = 0;
    if (!r.dataset(g + "counts", &dims, &kind, nullptr, 0)) return io_fail(LCS_EINVAL, r.err);
    if (dims.size() != 1 || dims[0] != 1 || kind != 'i')  // load.jl:75-77: one count per rank
      return io_fail(LCS_EINVAL, g + "counts: the file was written by " +
                                     std::to_string(dims.empty() ? 0 : dims[0]) + " ranks, expected 1");
    int64_t cnt = 0;
    if (!r.dataset(g + "counts", &dims, &kind, &cnt, 8)) return io_fail(LCS_EINVAL, r.err);
    if (cnt != n)
      return io_fail(LCS_EINVAL, g + "counts: " + std::to_string(cnt) + " particles, the handle holds " +
                                     std::to_string(n));
    std::vector<int64_t> ids((size_t)n);
    std::vector<std::vector<double>> pr(7, std::vector<double>((size_t)n));
    if (!r.dataset(g + "id", &dims, &kind, ids.data(), (uint64_t)n * 8)) return io_fail(LCS_EINVAL, r.err);
    for (int q = 0; q < 7; q++)
      if (!r.dataset(g + kProp[q], &dims, &kind, pr[q].data(), (uint64_t)n * 8)) return io_fail(LCS_EINVAL, r.err);
    rc = lcs_upload_particles(h, s, n, ids.data(), pr[0].data(), pr[1].data(), pr[2].data(), pr[3].data(),
                              pr[4].data(), pr[5].data(), pr[6].data());
    if (rc != LCS_OK) return handle_rc(h, rc);
  }
  return LCS_OK;
}

int lcs_restart_load_coarse(lcs_handle* h, const char* path) {
  if (!h || !path) return io_fail(LCS_EINVAL, "null argument");
  lcs_config c;
  if (lcs_get_config(h, &c) != LCS_OK) return io_fail(LCS_EINVAL, "bad handle");
  const lcs_config* cfg = &c;
  if (cfg->dims[0] % 2 || cfg->dims[1] % 2 || cfg->dims[2] % 2) return io_fail(LCS_EINVAL, "upsampling needs even dims");
  Reader r;
  if (!r.open(path)) return io_fail(LCS_EINVAL, r.err);
  return load_flow(h, r, cfg->dims[0] / 2, cfg->dims[1] / 2, cfg->dims[2] / 2, true);
}

// A save of one step of the stat file.  The reference opens the file "cw" and
// replaces the step's group (save.jl:17-31); this writer makes whole files, so
// an existing file is read whole, every entry outside the top-level group
// `<step>` is kept, and the file is written again under a temporary name that
// then replaces it.  A file this reader cannot read is left as it is (error).
struct StatFile {
  Writer w;
  std::vector<Reader::Item> kept;
  std::deque<double> f;  // storage of the new scalars and arrays
  std::deque<int64_t> i;
  std::deque<std::vector<double>> fa;
  std::deque<std::vector<int64_t>> ia;
  int open(const char* path, const std::string& step) {
    if (FILE* t = fopen(path, "rb")) {
      fclose(t);
      Reader r;
      if (!r.open(path) || !r.walk(r.root_oh, "", &kept, 0))
        return io_fail(LCS_EINVAL, std::string(path) + ": " + r.err + " (the file is left unchanged)");
    }
    for (auto& it : kept) {
      if (it.path == step || it.path.compare(0, step.size() + 1, step + "/") == 0) continue;
      const size_t q = it.path.rfind('/');
      const std::string g = q == std::string::npos ? "" : it.path.substr(0, q);
      const std::string name = q == std::string::npos ? it.path : it.path.substr(q + 1);
      if (it.group)
        w.group(it.path);
      else
        w.dataset(g, name, it.kind, it.dims, it.data.data());
    }
    return LCS_OK;
  }
  void scalar(const std::string& g, const std::string& name, double v) {
    f.push_back(v);
    w.dataset(g, name, 'f', {}, &f.back());
  }
  void scalar_i(const std::string& g, const std::string& name, int64_t v) {
    i.push_back(v);
    w.dataset(g, name, 'i', {}, &i.back());
  }
  void array(const std::string& g, const std::string& name, const double* v, size_t n) {  // empty: not written
    if (!n) return;
    fa.emplace_back(v, v + n);
    w.dataset(g, name, 'f', {(uint64_t)n}, fa.back().data());
  }
  void array_i(const std::string& g, const std::string& name, const int64_t* v, size_t n) {
    if (!n) return;
    ia.emplace_back(v, v + n);
    w.dataset(g, name, 'i', {(uint64_t)n}, ia.back().data());
  }
  void summary(const std::string& g, const lcs_summary& m) {  // LCS.Summary (src/stat.jl:4-9)
    scalar(g, "mean", m.mean);
    scalar(g, "max", m.max);
    scalar(g, "min", m.min);
  }
  int write(const char* path) {
    const std::string tmp = std::string(path) + ".tmp";
    const int rc = w.write(tmp.c_str());
    if (rc != LCS_OK) {
      remove(tmp.c_str());
      return rc;
    }
    if (rename(tmp.c_str(), path) != 0) {
      remove(tmp.c_str());
      return io_fail(LCS_EINVAL, std::string("cannot replace ") + path);
    }
    return LCS_OK;
  }
};

int lcs_stat_state_save(const char* path, int64_t step, double t, double dt) {
  if (!path) return io_fail(LCS_EINVAL, "null path");
  const std::string key = std::to_string(step);
  StatFile sf;
  if (int rc = sf.open(path, key)) return rc;
  sf.scalar_i(key + "/state", "step", step);
  sf.scalar(key + "/state", "t", t);
  sf.scalar(key + "/state", "dt", dt);
  return sf.write(path);
}

// One `<step>` entry of the stat file as LCSIO.savestat writes it
// (save.jl:1-33): Utils.deepwrite (src/utils/hdf5.jl:5-19) of the normalized
// State, Stat and log, with the Julia field names as dataset names.
int lcs_stat_save(const char* path, int64_t step, double t, double dt, const lcs_flow_stats* fs, int32_t ns,
                  const int64_t* nvalid, const lcs_particle_stats* ps, const lcs_log* lg) {
  if (!path) return io_fail(LCS_EINVAL, "null path");
  if (ns < 0 || ns > LCS_MAX_SPECIES) return io_fail(LCS_EINVAL, "species count out of range");
  for (int32_t s = 0; ps && s < ns; s++)
    if (ps[s].nbins < 0 || ps[s].nbins > LCS_RDF_MAX_BINS || ps[s].nshells < 0 ||
        ps[s].nshells > LCS_SPECTRUM_MAX_SHELLS)
      return io_fail(LCS_EINVAL, "species " + std::to_string(s) + ": bin or shell count out of range");
  const std::string key = std::to_string(step);
  StatFile sf;
  if (int rc = sf.open(path, key)) return rc;
  // state: LCS.State (src/state.jl:15-22); FlowState has no fields,
  // ParticleState holds nvalid (src/particles/state.jl:6-8)
  const std::string st = key + "/state";
  sf.scalar_i(st, "step", step);
  sf.scalar(st, "t", t);
  sf.scalar(st, "dt", dt);
  for (int32_t s = 0; nvalid && s < ns; s++) sf.scalar_i(st + "/particles/" + std::to_string(s + 1), "nvalid", nvalid[s]);
  // stat: LCS.Stat (src/stat.jl:26-40) = StateStat, FlowStat, ParticleStat...
  const std::string ss = key + "/stat";
  sf.scalar_i(ss + "/state", "step", step);
  sf.scalar(ss + "/state", "t", t);
  sf.scalar(ss + "/state", "dt", dt);
  if (fs) {  // FlowStat (src/flows/stat.jl:22-39)
    const std::string g = ss + "/flow";
    sf.summary(g + "/u", lcs_summary{fs->u_mean, fs->u_max, fs->u_min});
    sf.summary(g + "/v", lcs_summary{fs->v_mean, fs->v_max, fs->v_min});
    sf.summary(g + "/w", lcs_summary{fs->w_mean, fs->w_max, fs->w_min});
    sf.scalar(g, "k", fs->k);
    sf.scalar(g, "\u03F5", fs->epsilon);           // ϵ
    sf.scalar(g, "\u03C4\u03B7", fs->tau_eta);      // τη
    sf.scalar(g, "l\u03BC", fs->l_mu);              // lμ
    sf.scalar(g, "l\u03B7", fs->l_eta);             // lη
    sf.scalar(g, "Re\u03BB", fs->Re_lambda);        // Reλ
    sf.scalar(g, "urms", fs->urms);
    sf.scalar(g, "k\u03B7", fs->k_eta);             // kη
    sf.scalar(g, "skew", fs->skewness);
    sf.scalar(g, "flat", fs->flatness);
    sf.scalar(g, "L", fs->L);
    sf.scalar(g, "C\u03F5", fs->C_epsilon);         // Cϵ
  }
  for (int32_t s = 0; ps && s < ns; s++) {  // ParticleStat, RDFStat, SpectrumStat (src/particles/stat.jl:10-77)
    const lcs_particle_stats& p = ps[s];
    const std::string g = ss + "/particles/" + std::to_string(s + 1);
    sf.summary(g + "/x", p.x);
    sf.summary(g + "/y", p.y);
    sf.summary(g + "/z", p.z);
    sf.summary(g + "/u", p.u);
    sf.summary(g + "/v", p.v);
    sf.summary(g + "/w", p.w);
    sf.summary(g + "/diam", p.diam);
    sf.scalar(g, "\u03C4p", p.taup);                // τp
    sf.scalar(g, "St", p.St);
    sf.scalar(g + "/rdf", "gr_contact", p.gr_contact);
    sf.scalar_i(g + "/rdf", "npairs_contact", p.npairs_contact);
    if (p.nbins > 0) sf.array(g + "/rdf", "edges", p.edges, (size_t)p.nbins + 1);
    sf.array(g + "/rdf", "gr", p.gr, (size_t)p.nbins);
    sf.array_i(g + "/rdf", "npairs", p.npairs, (size_t)p.nbins);
    sf.array(g + "/spectrum", "wavenumbers", p.wavenumbers, (size_t)p.nshells);
    sf.array(g + "/spectrum", "Enp", p.Enp, (size_t)p.nshells);
  }
  if (lg) {  // the step's evolve! log (src/evolve.jl:126-145): the couples' (; itr, div), the forcing's (; p[, e10])
    const std::string g = key + "/log/flow";
    sf.scalar_i(g + "/couple1", "itr", lg->couple1.itr);
    sf.scalar(g + "/couple1", "div", lg->couple1.div);
    sf.scalar_i(g + "/couple2", "itr", lg->couple2.itr);
    sf.scalar(g + "/couple2", "div", lg->couple2.div);
    if (!std::isnan(lg->forcing_p)) sf.scalar(g + "/forcing", "p", lg->forcing_p);
    if (!std::isnan(lg->forcing_e10)) sf.scalar(g + "/forcing", "e10", lg->forcing_e10);
  }
  return sf.write(path);
}

int lcs_stat_state_load(const char* path, int64_t step, double* t, double* dt) {
  if (!path) return io_fail(LCS_EINVAL, "null path");
  Reader r;
  if (!r.open(path)) return io_fail(LCS_EINVAL, r.err);
  const std::string g = std::to_string(step) + "/state/";
  std::vector<uint64_t> dims;
  char kind = 0;
  if (t && !r.dataset(g + "t", &dims, &kind, t, 8)) return io_fail(LCS_EINVAL, r.err);
  if (dt && !r.dataset(g + "dt", &dims, &kind, dt, 8)) return io_fail(LCS_EINVAL, r.err);
  return LCS_OK;
}

// Inspection of any file of the supported subset: the dims and kind of a
// dataset, and its data when buf is given (bytes = 8 x element count).
int lcs_h5_dataset(const char* path, const char* name, int32_t* rank, int64_t* dims, char* kind, void* buf,
                   int64_t bytes) {
  if (!path || !name || !rank || !dims || !kind) return io_fail(LCS_EINVAL, "null argument");
  Reader r;
  if (!r.open(path)) return io_fail(LCS_EINVAL, r.err);
  std::vector<uint64_t> d;
  if (!r.dataset(name, &d, kind, nullptr, 0)) return io_fail(LCS_EINVAL, r.err);
  if (d.size() > 8) return io_fail(LCS_EINVAL, "rank above 8");
  *rank = (int32_t)d.size();
  for (size_t q = 0; q < d.size(); q++) dims[q] = (int64_t)d[q];
  if (buf && !r.dataset(name, &d, kind, buf, (uint64_t)bytes)) return io_fail(LCS_EINVAL, r.err);
  return LCS_OK;
}
// Names in a group ("" or "/" for the root), as one string of '\n'-separated
// names (sorted), written into buf (cap bytes, truncated).
int lcs_h5_list(const char* path, const char* group, char* buf, int64_t cap) {
  if (!path || !group || !buf || cap < 1) return io_fail(LCS_EINVAL, "null argument");
  Reader r;
  if (!r.open(path)) return io_fail(LCS_EINVAL, r.err);
  uint64_t oh;
  if (!r.find(group, &oh)) return io_fail(LCS_EINVAL, r.err);
  std::map<std::string, uint64_t> ch;
  if (!r.children(oh, &ch)) return io_fail(LCS_EINVAL, r.err);
  std::string s;
  for (auto& kv : ch) s += kv.first + "\n";
  snprintf(buf, (size_t)cap, "%s", s.c_str());
  return LCS_OK;
}

}  // extern "C"
