// gpulda_train.cpp -- C++ twin of the reference's Rust training driver
// (src/train.rs:14-105 with src/buffer.rs and src/ffi.rs), which cannot be
// built here (no Rust toolchain).  It makes the same calls through the same C
// ABI in the same order:
//   initialize(&args, buffers, 1)
//   repeat n_mc times: sample_phi(); for each filled buffer:
//       sample_z_async(b); sync_buffer(b); advance
//   cleanup(buffers, 1)
// over memory-mapped z.bin (read-write), w.bin, d.bin, k_d.bin (read-only) and
// the word counts in the third column of c.txt.
//
// Flags follow src/args.rs:17-59 (same names and defaults).  --seed is passed
// to the library through gpulda_initialize_ex; the reference parses it but
// never forwards it (its CUDA side uses seed 0, which is also the default here).
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "gpulda.h"

namespace {

struct Options {
  float alpha = 0.1f, beta = 0.1f;
  uint32_t K = 100, buffer_size = 33554432, max_D = 16384, n_mc = 1, seed = 0;
  std::string z = "temp/z.bin", w = "temp/w.bin", d = "temp/d.bin", k_d = "temp/k_d.bin", c = "temp/c.txt";
};

struct Map {
  uint8_t* p = nullptr;
  size_t n = 0;
};

Map map_file(const std::string& path, bool writable) {
  const int fd = open(path.c_str(), writable ? O_RDWR : O_RDONLY);
  if (fd < 0) {
    fprintf(stderr, "cannot open %s\n", path.c_str());
    exit(1);
  }
  struct stat st;
  fstat(fd, &st);
  Map m;
  m.n = (size_t)st.st_size;
  if (m.n) {
    void* p = mmap(nullptr, m.n, writable ? PROT_READ | PROT_WRITE : PROT_READ, MAP_SHARED, fd, 0);
    if (p == MAP_FAILED) {
      fprintf(stderr, "cannot map %s\n", path.c_str());
      exit(1);
    }
    m.p = (uint8_t*)p;
  }
  close(fd);
  return m;
}

// src/train.rs:15-18: third tab-separated column of c.txt.
std::vector<uint32_t> token_counts(const std::string& path) {
  std::ifstream f(path);
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
  Map m;
  size_t pos = 0;
  bool read_u32(uint32_t* v) {
    if (pos + 4 > m.n) return false;
    std::memcpy(v, m.p + pos, 4);
    pos += 4;
    return true;
  }
};

// src/train.rs:20-47: take documents while the next length is nonzero, at most
// max_D documents and buffer_size tokens.
void fill_buffer(Buffer& b, Cursor& z, Cursor& w, Cursor& d, Cursor& k_d, const Options& o) {
  const size_t orig = d.pos;
  uint32_t n_docs = 0, n_tokens = 0;
  while (true) {
    uint32_t sz = 0;
    if (!d.read_u32(&sz)) sz = 0;
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
  d.pos = orig;
  b.n_docs = n_docs;
  b.n_tokens = n_tokens;
  b.z = (uint32_t*)(z.m.p + z.pos);
  b.w = (uint32_t*)(w.m.p + w.pos);
  b.d = (uint32_t*)(d.m.p + d.pos);
  b.K_d = (uint32_t*)(k_d.m.p + k_d.pos);
}

// src/train.rs:49-58.
void empty_buffer(Buffer& b, Cursor& z, Cursor& w, Cursor& d, Cursor& k_d) {
  z.pos += (size_t)b.n_tokens * 4;
  w.pos += (size_t)b.n_tokens * 4;
  d.pos += (size_t)b.n_docs * 4;
  k_d.pos += (size_t)b.n_docs * 4;
  b.n_docs = 0;
  b.n_tokens = 0;
}

bool parse(int argc, char** argv, Options& o) {
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
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
    else if (a == "--z_temp_file") o.z = val();
    else if (a == "--w_temp_file") o.w = val();
    else if (a == "--d_temp_file") o.d = val();
    else if (a == "--K_d_temp_file") o.k_d = val();
    else if (a == "--c_temp_file") o.c = val();
    else {
      fprintf(stderr, "unknown flag %s\n", a.c_str());
      return false;
    }
  }
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  Options o;
  if (!parse(argc, argv, o)) return 2;
  printf("training\n");
  std::vector<uint32_t> c = token_counts(o.c);
  Args args{o.alpha, o.beta, o.K, (uint32_t)c.size(), c.data(), o.buffer_size, o.max_D};
  std::vector<Buffer> buffers(1);
  std::memset(buffers.data(), 0, sizeof(Buffer));
  GpuldaExArgs ex{o.seed, 0, 0};
  gpulda_set_fatal_errors(1);
  if (gpulda_initialize_ex(&args, buffers.data(), 1, &ex) != GPULDA_OK) {
    fprintf(stderr, "initialize failed\n");
    return 1;
  }
  Cursor z{map_file(o.z, true)}, w{map_file(o.w, false)}, d{map_file(o.d, false)}, k_d{map_file(o.k_d, false)};
  for (uint32_t it = 0; it < o.n_mc; ++it) {
    sample_phi();
    bool done = false;
    while (!done) {
      for (Buffer& b : buffers) {
        fill_buffer(b, z, w, d, k_d, o);
        if (b.n_docs == 0) {
          done = true;
          break;
        }
        sample_z_async(&b);
        sync_buffer(&b);
        empty_buffer(b, z, w, d, k_d);
      }
    }
    if (z.m.p) msync(z.m.p, z.m.n, MS_SYNC);
    z.pos = w.pos = d.pos = k_d.pos = 0;
    printf("finished iteration: %u\n", it);
  }
  cleanup(buffers.data(), 1);
  return 0;
}
