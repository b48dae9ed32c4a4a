// gpulda_train.cpp -- C++ twin of the reference's Rust command line
// (src/main.rs: preprocess, train, output), which cannot be built here (no
// Rust toolchain).
//
//   preprocess (src/preprocess.rs:16-72): token counts of the input's third
//     tab-separated field, ids ranked by descending count into c.txt
//     ("token<TAB>id<TAB>count"); per document its topics z (uniform initial
//     topics), word ids w, length d and number of distinct initial topics K_d,
//     as u32 binary files.
//   train (src/train.rs:14-105 with src/buffer.rs and src/ffi.rs): the same
//     calls through the same C ABI in the same order --
//       initialize(&args, buffers, n)
//       repeat n_mc times: sample_phi(); for each filled buffer:
//           sample_z_async(b); sync_buffer(b); advance
//       cleanup(buffers, n)
//     over memory-mapped z.bin (read-write), w.bin, d.bin, k_d.bin
//     (read-only) and the counts of c.txt.
//   output (src/output.rs:27-62): one line per document of "token:topic<TAB>"
//     pairs.
//
// Flags follow src/args.rs:17-59 (same names and defaults).  --seed reaches
// the sampler through gpulda_initialize_ex (the reference parses it but never
// forwards it) and seeds the initial topics of preprocess (the reference uses
// an unseeded generator).  Additions: --phases (comma list, default all three
// as main.rs runs them), --double_buffer 1 (two buffers in flight: the next
// buffer's copies and sweep are issued before the previous one is waited for;
// the result is identical) and --pin 1 (page-lock the mapped files so the
// buffer copies are asynchronous DMA), for corpora streamed from files that
// are larger than device memory.
//
// Deliberate differences: word ids with equal counts are ranked by first
// occurrence in the input (the reference's order among equal counts comes
// from hash-map iteration and is arbitrary); a line without a third field is
// reported as an error with its line number (the reference panics).
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "gpulda.h"

namespace {

struct Options {
  float alpha = 0.1f, beta = 0.1f;
  uint32_t K = 100, buffer_size = 33554432, max_D = 16384, n_mc = 1, seed = 0;
  std::string input = "data/small.txt", output = "output/small.txt";
  std::string z = "temp/z.bin", w = "temp/w.bin", d = "temp/d.bin", k_d = "temp/k_d.bin", c = "temp/c.txt";
  std::string phases = "preprocess,train,output";
  bool double_buffer = false, pin = false;
};

[[noreturn]] void die(const std::string& what) {
  fprintf(stderr, "%s\n", what.c_str());
  exit(1);
}

// ---- preprocess (src/preprocess.rs) --------------------------------------

// The third tab-separated field, split on whitespace (src/preprocess.rs:12-14).
bool tokens_of(const std::string& line, std::vector<std::string>& out) {
  out.clear();
  size_t a = line.find('\t');
  if (a == std::string::npos) return false;
  size_t b = line.find('\t', a + 1);
  if (b == std::string::npos) return false;
  size_t e = line.find('\t', b + 1);
  const std::string field = line.substr(b + 1, e == std::string::npos ? std::string::npos : e - b - 1);
  std::istringstream ss(field);
  std::string t;
  while (ss >> t) out.push_back(t);
  return true;
}

// splitmix64: seeded initial topics.
struct Rng {
  uint64_t s;
  uint64_t next() {
    uint64_t x = (s += 0x9E3779B97F4A7C15ull);
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
  }
  uint32_t below(uint32_t K) { return (uint32_t)(((next() >> 32) * (uint64_t)K) >> 32); }
};

void write_u32(FILE* f, const uint32_t* v, size_t n) {
  if (n && fwrite(v, 4, n, f) != n) die("write failed");
}

void preprocess(const Options& o) {
  printf("preprocessing\n");
  // src/preprocess.rs:16-32: counts, ids by descending count
  std::unordered_map<std::string, std::pair<uint32_t, uint32_t>> count;  // token -> (count, first seen)
  std::vector<std::string> toks;
  {
    std::ifstream in(o.input);
    if (!in) die("cannot open input " + o.input);
    std::string line;
    size_t ln = 0;
    uint32_t order = 0;
    while (std::getline(in, line)) {
      ++ln;
      if (!tokens_of(line, toks)) die("line " + std::to_string(ln) + " of " + o.input + " has no token field");
      for (auto& t : toks) {
        auto it = count.find(t);
        if (it == count.end())
          count.emplace(t, std::make_pair(1u, order++));
        else
          ++it->second.first;
      }
    }
  }
  std::vector<std::pair<std::string, std::pair<uint32_t, uint32_t>>> ranked(count.begin(), count.end());
  std::sort(ranked.begin(), ranked.end(), [](const auto& x, const auto& y) {
    return x.second.first != y.second.first ? x.second.first > y.second.first : x.second.second < y.second.second;
  });
  std::unordered_map<std::string, uint32_t> ids;
  ids.reserve(ranked.size());
  {
    FILE* c = fopen(o.c.c_str(), "w");
    if (!c) die("cannot create " + o.c);
    for (size_t i = 0; i < ranked.size(); ++i) {
      fprintf(c, "%s\t%zu\t%u\n", ranked[i].first.c_str(), i, ranked[i].second.first);
      ids[ranked[i].first] = (uint32_t)i;
    }
    fclose(c);
  }
  // src/preprocess.rs:43-72: per document z, w, d, k_d
  FILE* fz = fopen(o.z.c_str(), "wb");
  FILE* fw = fopen(o.w.c_str(), "wb");
  FILE* fd = fopen(o.d.c_str(), "wb");
  FILE* fk = fopen(o.k_d.c_str(), "wb");
  if (!fz || !fw || !fd || !fk) die("cannot create the temporary files");
  Rng rng{o.seed};
  std::ifstream in(o.input);
  std::string line;
  std::vector<uint32_t> z, w;
  while (std::getline(in, line)) {
    tokens_of(line, toks);
    z.resize(toks.size());
    w.resize(toks.size());
    for (size_t i = 0; i < toks.size(); ++i) {
      z[i] = rng.below(o.K);
      w[i] = ids[toks[i]];
    }
    write_u32(fz, z.data(), z.size());
    write_u32(fw, w.data(), w.size());
    const uint32_t L = (uint32_t)toks.size();
    write_u32(fd, &L, 1);
    std::sort(z.begin(), z.end());
    const uint32_t kd = (uint32_t)(std::unique(z.begin(), z.end()) - z.begin());
    write_u32(fk, &kd, 1);
  }
  fclose(fz);
  fclose(fw);
  fclose(fd);
  fclose(fk);
}

// ---- train (src/train.rs) ----------------------------------------------------

struct Map {
  uint8_t* p = nullptr;
  size_t n = 0;
  bool pinned = false;
};

Map map_file(const std::string& path, bool writable) {
  const int fd = open(path.c_str(), writable ? O_RDWR : O_RDONLY);
  if (fd < 0) die("cannot open " + path);
  struct stat st;
  fstat(fd, &st);
  Map m;
  m.n = (size_t)st.st_size;
  if (m.n) {
    void* p = mmap(nullptr, m.n, writable ? PROT_READ | PROT_WRITE : PROT_READ, MAP_SHARED, fd, 0);
    if (p == MAP_FAILED) die("cannot map " + path);
    m.p = (uint8_t*)p;
  }
  close(fd);
  return m;
}

void pin(Map& m, bool read_only) {
  if (!m.p) return;
  gpulda_set_fatal_errors(0);
  m.pinned = gpulda_pin_host(m.p, m.n, read_only ? GPULDA_PIN_READ_ONLY : 0u) == GPULDA_OK;
  gpulda_set_fatal_errors(1);
  if (!m.pinned) fprintf(stderr, "note: could not pin a mapped file; copies are staged instead\n");
}

void unmap(Map& m) {
  if (m.pinned) gpulda_unpin_host(m.p);
  if (m.p) munmap(m.p, m.n);
  m = Map();
}

// src/train.rs:15-18: third tab-separated column of c.txt.
std::vector<uint32_t> token_counts(const std::string& path) {
  std::ifstream f(path);
  if (!f) die("cannot open " + path);
  std::vector<uint32_t> c;
  std::string line;
  while (std::getline(f, line)) {
    std::stringstream ss(line);
    std::string a, b, cnt;
    std::getline(ss, a, '\t');
    std::getline(ss, b, '\t');
    std::getline(ss, cnt, '\t');
    c.push_back((uint32_t)std::stoul(cnt));
  }
  return c;
}

struct Cursor {
  Map* m;
  size_t pos = 0;
  bool read_u32(size_t at, uint32_t* v) const {
    if (at + 4 > m->n) return false;
    std::memcpy(v, m->p + at, 4);
    return true;
  }
};

// src/train.rs:20-47: take documents while the next length is nonzero, at most
// max_D documents and buffer_size tokens; then advance past them (the
// reference advances in empty_buffer, src/train.rs:49-58, after the sync).
void fill_buffer(Buffer& b, Cursor& z, Cursor& w, Cursor& d, Cursor& k_d, const Options& o) {
  uint32_t n_docs = 0, n_tokens = 0;
  size_t at = d.pos;
  while (true) {
    uint32_t sz = 0;
    if (!d.read_u32(at, &sz)) sz = 0;
    at += 4;
    n_docs += 1;
    n_tokens += sz;
    if (sz > o.buffer_size) {
      fprintf(stderr, "document size exceeded buffer size: %u\n", sz);
      exit(101);
    }
    if (sz == 0 || n_docs > o.max_D || n_tokens > o.buffer_size) {
      n_docs -= 1;
      n_tokens -= sz;
      break;
    }
  }
  b.n_docs = n_docs;
  b.n_tokens = n_tokens;
  b.z = (uint32_t*)(z.m->p + z.pos);
  b.w = (uint32_t*)(w.m->p + w.pos);
  b.d = (uint32_t*)(d.m->p + d.pos);
  b.K_d = (uint32_t*)(k_d.m->p + k_d.pos);
  z.pos += (size_t)n_tokens * 4;
  w.pos += (size_t)n_tokens * 4;
  d.pos += (size_t)n_docs * 4;
  k_d.pos += (size_t)n_docs * 4;
}

void train(const Options& o) {
  printf("training\n");
  std::vector<uint32_t> c = token_counts(o.c);
  const uint32_t nb = o.double_buffer ? 2 : 1;
  Args args{o.alpha, o.beta, o.K, (uint32_t)c.size(), c.data(), o.buffer_size, o.max_D};
  std::vector<Buffer> buffers(nb);
  std::memset(buffers.data(), 0, nb * sizeof(Buffer));
  GpuldaExArgs ex{o.seed, 0, 0};
  gpulda_set_fatal_errors(1);
  if (gpulda_initialize_ex(&args, buffers.data(), nb, &ex) != GPULDA_OK) die("initialize failed");
  Map mz = map_file(o.z, true), mw = map_file(o.w, false), md = map_file(o.d, false), mk = map_file(o.k_d, false);
  if (o.pin) {
    pin(mz, false);
    pin(mw, true);
    pin(md, true);
    pin(mk, true);
  }
  Cursor z{&mz}, w{&mw}, d{&md}, k_d{&mk};
  for (uint32_t it = 0; it < o.n_mc; ++it) {
    sample_phi();
    if (!o.double_buffer) {
      while (true) {  // src/train.rs:92-100
        Buffer& b = buffers[0];
        fill_buffer(b, z, w, d, k_d, o);
        if (b.n_docs == 0) break;
        sample_z_async(&b);
        sync_buffer(&b);
      }
    } else {
      // buffer i+1 is filled and submitted before buffer i is waited for
      uint32_t cur = 0;
      fill_buffer(buffers[cur], z, w, d, k_d, o);
      if (buffers[cur].n_docs) sample_z_async(&buffers[cur]);
      while (buffers[cur].n_docs) {
        Buffer& nx = buffers[cur ^ 1];
        fill_buffer(nx, z, w, d, k_d, o);
        if (nx.n_docs) sample_z_async(&nx);
        sync_buffer(&buffers[cur]);
        cur ^= 1;
      }
    }
    if (mz.p) msync(mz.p, mz.n, MS_SYNC);
    z.pos = w.pos = d.pos = k_d.pos = 0;
    printf("finished iteration: %u\n", it);
  }
  cleanup(buffers.data(), nb);
  unmap(mz);
  unmap(mw);
  unmap(md);
  unmap(mk);
}

// ---- output (src/output.rs) ---------------------------------------------------

void output(const Options& o) {
  printf("writing output\n");
  std::vector<std::string> names;
  {
    std::ifstream f(o.c);
    if (!f) die("cannot open " + o.c);
    std::string line;
    while (std::getline(f, line)) {
      const size_t a = line.find('\t');
      const size_t b = line.find('\t', a + 1);
      if (a == std::string::npos || b == std::string::npos) die("malformed line in " + o.c);
      const size_t id = std::stoul(line.substr(a + 1, b - a - 1));
      if (names.size() <= id) names.resize(id + 1);
      names[id] = line.substr(0, a);
    }
  }
  Map mz = map_file(o.z, false), mw = map_file(o.w, false), md = map_file(o.d, false);
  FILE* out = fopen(o.output.c_str(), "w");
  if (!out) die("cannot create " + o.output);
  const uint32_t* z = (const uint32_t*)mz.p;
  const uint32_t* w = (const uint32_t*)mw.p;
  const uint32_t* d = (const uint32_t*)md.p;
  const size_t n_docs = md.n / 4, n_tok = std::min(mz.n, mw.n) / 4;
  size_t pos = 0;
  for (size_t i = 0; i < n_docs; ++i) {
    for (uint32_t j = 0; j < d[i] && pos < n_tok; ++j, ++pos) {
      if (w[pos] >= names.size()) die("word id beyond c.txt in " + o.w);
      fprintf(out, "%s:%u\t", names[w[pos]].c_str(), z[pos]);
    }
    fputc('\n', out);
  }
  fclose(out);
  unmap(mz);
  unmap(mw);
  unmap(md);
}

// The flags of src/args.rs:16-61 with their defaults, plus this twin's own.
void usage(FILE* f) {
  const Options d;
  fprintf(f,
          "gpulda_train: preprocess, train and output as the reference's command line does\n"
          "  --alpha F          alpha parameter (%g)\n"
          "  --beta F           beta parameter (%g)\n"
          "  --K N              number of topics (%u)\n"
          "  --buffer_size N    tokens per buffer (%u)\n"
          "  --max_D N          documents per buffer (%u)\n"
          "  --n_mc N           Gibbs iterations (%u)\n"
          "  --seed N           random number seed (%u)\n"
          "  --input PATH       corpus text (%s)\n"
          "  --output PATH      token:topic output (%s)\n"
          "  --z_temp_file, --w_temp_file, --d_temp_file, --K_d_temp_file PATH   u32 binaries (%s, %s, %s, %s)\n"
          "  --c_temp_file PATH word counts, one per line (%s)\n"
          "  --phases LIST      comma-separated subset of preprocess,train,output (%s)\n"
          "  --double_buffer 0|1  two buffers in flight (%d)\n"
          "  --pin 0|1          page-lock the mapped files (%d)\n",
          d.alpha, d.beta, d.K, d.buffer_size, d.max_D, d.n_mc, d.seed, d.input.c_str(), d.output.c_str(),
          d.z.c_str(), d.w.c_str(), d.d.c_str(), d.k_d.c_str(), d.c.c_str(), d.phases.c_str(), (int)d.double_buffer,
          (int)d.pin);
}

bool parse(int argc, char** argv, Options& o) {
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if (a == "--help" || a == "-h") {
      usage(stdout);
      exit(0);
    }
    auto val = [&](void) -> std::string {
      if (i + 1 >= argc) {
        fprintf(stderr, "missing value for %s\n", a.c_str());
        exit(2);
      }
      return argv[++i];
    };
    if (a == "--alpha") o.alpha = std::stof(val());
    else if (a == "--beta") o.beta = std::stof(val());
    else if (a == "--K") o.K = (uint32_t)std::stoul(val());
    else if (a == "--buffer_size") o.buffer_size = (uint32_t)std::stoul(val());
    else if (a == "--max_D") o.max_D = (uint32_t)std::stoul(val());
    else if (a == "--n_mc") o.n_mc = (uint32_t)std::stoul(val());
    else if (a == "--seed") o.seed = (uint32_t)std::stoul(val());
    else if (a == "--input") o.input = val();
    else if (a == "--output") o.output = val();
    else if (a == "--z_temp_file") o.z = val();
    else if (a == "--w_temp_file") o.w = val();
    else if (a == "--d_temp_file") o.d = val();
    else if (a == "--K_d_temp_file") o.k_d = val();
    else if (a == "--c_temp_file") o.c = val();
    else if (a == "--phases") o.phases = val();
    else if (a == "--double_buffer") o.double_buffer = std::stoul(val()) != 0;
    else if (a == "--pin") o.pin = std::stoul(val()) != 0;
    else {
      fprintf(stderr, "unknown flag %s\n", a.c_str());
      usage(stderr);
      return false;
    }
  }
  return true;
}

bool has_phase(const std::string& phases, const char* p) {
  std::stringstream ss(phases);
  std::string t;
  while (std::getline(ss, t, ','))
    if (t == p) return true;
  return false;
}

}  // namespace

int main(int argc, char** argv) {
  Options o;
  if (!parse(argc, argv, o)) return 2;
  if (o.K < 1) die("--K must be positive");
  if (has_phase(o.phases, "preprocess")) preprocess(o);
  if (has_phase(o.phases, "train")) train(o);
  if (has_phase(o.phases, "output")) output(o);
  return 0;
}
