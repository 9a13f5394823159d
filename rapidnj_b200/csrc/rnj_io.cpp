// rnj_io.cpp -- host-side alignment reader and "-o m" matrix writer.
//
// The reader keeps the reference loaders' character rules so that the same file
// gives the same n x L byte matrix:
//   FASTA (dataloaderFasta.hpp:78-133,201-276): ';' lines are comments, '>'
//   starts a name (bytes > 31), every other line contributes its bytes > 32;
//   end of file reads as a newline.
//   Stockholm (dataloaderStockholm.hpp:79-120,185-307): bytes < 32 between lines
//   are skipped, '#' lines are markup, "//" ends the alignment (required), a
//   sequence line is a name (bytes > 32) followed by its residues (bytes > 32).
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "rnj.h"
#include "rnj_internal.h"
#include "rnj_objects.h"

using rnj::set_error;

namespace {

// The file's bytes: read into one uninitialised buffer (a zero-filled one would
// cost another pass over it), or a caller's buffer viewed in place.
struct FileData {
  std::unique_ptr<char[]> buf;
  const char *view = nullptr;
  size_t n = 0;
  size_t size() const { return n; }
  char operator[](size_t i) const { return data()[i]; }
  const char *data() const { return view ? view : buf.get(); }
};

bool read_file(const char *path, FileData &fd) {
  FILE *f = fopen(path, "rb");
  if (!f) return false;
  size_t cap = 0;
  if (fseek(f, 0, SEEK_END) == 0) {
    const long size = ftell(f);
    if (size > 0) cap = (size_t)size;
  }
  rewind(f);
  cap = std::max<size_t>(cap, 1 << 16);
  fd.buf.reset(new char[cap]);
  fd.n = 0;
  while (true) {
    if (fd.n == cap) {  // the file grew, or its size was unknown
      std::unique_ptr<char[]> bigger(new char[2 * cap]);
      memcpy(bigger.get(), fd.buf.get(), fd.n);
      fd.buf.swap(bigger);
      cap *= 2;
    }
    const size_t k = fread(fd.buf.get() + fd.n, 1, cap - fd.n, f);
    if (k == 0) break;
    fd.n += k;
  }
  fclose(f);
  return true;
}

bool ends_with(const std::string &s, const char *suffix) {
  const size_t k = strlen(suffix);
  return s.size() >= k && s.compare(s.size() - k, k, suffix) == 0;
}

struct Builder {
  rnj_msa *m;
  bool first = true;
  int store(std::vector<char> &buf) {
    if (buf.empty()) return RNJ_OK;
    if (first) {
      m->L = (int)buf.size();
      m->type = rnj_detect_type(buf.data(), m->L);
      first = false;
    } else if ((int)buf.size() != m->L) {
      return set_error(RNJ_ERR_FORMAT, "ERROR: Sequence " + std::to_string(m->n) + " has length " +
                                           std::to_string(buf.size()) +
                                           " while the preceding sequences in the alignment which "
                                           "have length " + std::to_string(m->L) + ".");
    }
    m->chars.insert(m->chars.end(), buf.begin(), buf.end());
    m->n++;
    buf.clear();
    return RNJ_OK;
  }
};

// FASTA in whole lines: a line is found with memchr, a sequence line whose
// bytes are all > 32 (the common case) is appended with one copy, any other
// sequence line byte by byte with the reference's filter (signed chars > 32
// kept: control bytes, spaces and bytes >= 128 are dropped).  A name is the
// bytes > 31 after '>' up to the first other byte (dataloaderFasta.hpp:78-133).
int parse_fasta(const FileData &data, rnj_msa *m) {
  const char *p = data.data(), *end = p + data.size();
  // Sequences expected: the '>' that start a line.
  size_t headers = (p < end && *p == '>') ? 1 : 0;
  for (const char *q = p; q < end;) {
    const char *nl = (const char *)memchr(q, '\n', (size_t)(end - q));
    if (!nl) break;
    if (nl + 1 < end && nl[1] == '>') ++headers;
    q = nl + 1;
  }
  // The sequence being read is m->chars[seq0 ..): lines are appended there
  // directly and its length is checked when it ends.
  size_t seq0 = 0;
  bool first = true;
  auto finish = [&]() -> int {
    const size_t len = m->chars.size() - seq0;
    if (len == 0) return RNJ_OK;
    if (first) {
      m->L = (int)len;
      m->type = rnj_detect_type(m->chars.data() + seq0, m->L);
      first = false;
      m->chars.reserve(len * std::max<size_t>(headers, 1));
    } else if (len != (size_t)m->L) {
      return set_error(RNJ_ERR_FORMAT, "ERROR: Sequence " + std::to_string(m->n) + " has length " +
                                           std::to_string(len) +
                                           " while the preceding sequences in the alignment which "
                                           "have length " + std::to_string(m->L) + ".");
    }
    m->n++;
    seq0 = m->chars.size();
    return RNJ_OK;
  };
  auto append_seq = [&](const char *a, const char *z) {
    bool clean = true;
    for (const char *c = a; c < z; ++c) clean &= (signed char)*c > 32;
    if (clean) {
      m->chars.insert(m->chars.end(), a, z);
    } else {
      for (const char *c = a; c < z; ++c)
        if ((signed char)*c > 32) m->chars.push_back(*c);
    }
  };
  while (p < end) {
    const char *nl = (const char *)memchr(p, '\n', (size_t)(end - p));
    const char *le = nl ? nl : end;  // end of file reads as a newline
    // A segment of the line: the line itself, or what follows a name that
    // ended on a control byte before the newline (read as if a line began
    // there, as the reference's character loop does).
    for (const char *q = p; q < le;) {
      if (*q == ';') break;  // comment: the rest of the line
      if (*q == '>') {
        int rc = finish();
        if (rc != RNJ_OK) return rc;
        const char *a = q + 1, *c = a;
        while (c < le && (signed char)*c > 31) ++c;
        m->names.emplace_back(a, c);
        if (c >= le) break;
        q = c + 1;
        continue;
      }
      append_seq(q, le);
      break;
    }
    p = nl ? nl + 1 : end;
  }
  return finish();
}

int parse_stockholm(const FileData &data, rnj_msa *m) {
  size_t pos = 0;
  bool eof = false;
  auto next = [&]() -> char {
    if (pos < data.size()) return data[pos++];
    eof = true;
    return 0;
  };
  const char *truncated = "Stream ended unexpectedly. Did not find '//' marking the end of the alignment";
  Builder b{m};
  std::vector<char> buf;
  char c = next();
  while (true) {
    while (c < 32 && !eof) c = next();
    if (eof) return set_error(RNJ_ERR_FORMAT, truncated);
    std::string prefix;
    if (c == '#') {
      while (c != 10 && !eof) c = next();
    } else {
      if (c == '/') {
        c = next();
        if (c == '/') return RNJ_OK;
        prefix = "/";
      }
      std::string name = prefix;
      while (c > 32) {
        name.push_back(c);
        c = next();
      }
      m->names.push_back(name);
      while (c < 32 && !eof) {
        c = next();
        if (c == 10) return set_error(RNJ_ERR_FORMAT, "ERROR: alignment with name \"" + name + "\" has zero length");
      }
      while (c != 10 && !eof) {
        if (c > 32) buf.push_back(c);
        c = next();
      }
      int rc = b.store(buf);
      if (rc != RNJ_OK) return rc;
    }
    if (eof) return set_error(RNJ_ERR_FORMAT, truncated);
    c = next();
  }
}

// Six fixed decimals, as iostream's setprecision(6) << fixed prints a float
// (main.cpp:218): the float is widened to double and rounded to nearest.
inline int format_fixed6(char *out, float v) { return snprintf(out, 64, "%.6f ", (double)v); }

}  // namespace

// Parses bytes already in memory (the device reader's fallback for inputs its
// kernels leave to the host rules).
int msa_parse_buffer(const char *bytes, size_t size, bool fasta, rnj_msa *m) {
  FileData data;
  data.view = bytes;
  data.n = size;
  return fasta ? parse_fasta(data, m) : parse_stockholm(data, m);
}

int msa_format(const char *path, const char *format, bool *fasta) {
  std::string fmt = format ? format : "";
  std::string p(path);
  if (fmt.empty()) {
    if (ends_with(p, ".sth") || ends_with(p, ".STH")) fmt = "sth";
    else if (ends_with(p, ".fa") || ends_with(p, ".faa") || ends_with(p, ".fasta") ||
             ends_with(p, ".FA") || ends_with(p, ".FAA") || ends_with(p, ".FASTA"))
      fmt = "fa";
    else
      return set_error(RNJ_ERR_FORMAT, "ERROR: could not determine input file format. Please use "
                                        "the '-i' option to indicate the format.");
  }
  if (fmt != "fa" && fmt != "sth") return set_error(RNJ_ERR_UNSUPPORTED, "Unkown input format " + fmt);
  *fasta = fmt == "fa";
  return RNJ_OK;
}

extern "C" {

int rnj_msa_read(const char *path, const char *format, rnj_msa **out) {
  if (!path || !out) return set_error(RNJ_ERR_INVALID, "null argument");
  bool fasta = true;
  int rc = msa_format(path, format, &fasta);
  if (rc != RNJ_OK) return rc;
  FileData data;
  if (!read_file(path, data)) return set_error(RNJ_ERR_IO, std::string("ERROR: Could not read file: ") + path);
  rnj_msa *m = new rnj_msa();
  rc = fasta ? parse_fasta(data, m) : parse_stockholm(data, m);
  if (rc != RNJ_OK) {
    delete m;
    return rc;
  }
  *out = m;
  return RNJ_OK;
}

int rnj_msa_info(const rnj_msa *msa, int *n, int *L, int *detected_type) {
  if (!msa) return set_error(RNJ_ERR_INVALID, "null alignment");
  if (n) *n = msa->n;
  if (L) *L = msa->L;
  if (detected_type) *detected_type = msa->type;
  return RNJ_OK;
}

const char *rnj_msa_name(const rnj_msa *msa, int i) {
  if (!msa || i < 0 || i >= (int)msa->names.size()) return nullptr;
  return msa->names[i].c_str();
}

const char *rnj_msa_chars(const rnj_msa *msa) {
  if (!msa) return "";
  if (msa->chars.empty() && msa->d_chars && msa->n > 0 && msa->L > 0) {
    // An alignment read on the device: its bytes come to the host on first use.
    msa->chars.resize((size_t)msa->n * msa->L);
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != msa->device) cudaSetDevice(msa->device);
    const cudaError_t e = cudaMemcpy(msa->chars.data(), msa->d_chars, msa->chars.size(),
                                     cudaMemcpyDeviceToHost);
    if (prev >= 0 && prev != msa->device) cudaSetDevice(prev);
    if (e != cudaSuccess) {
      msa->chars.clear();
      rnj::cuda_error(e, "alignment download");
      return nullptr;
    }
  }
  return !msa->chars.empty() ? msa->chars.data() : "";
}

int rnj_msa_device_chars(const rnj_msa *msa, const void **d_chars, size_t *ld) {
  if (!msa || !d_chars) return set_error(RNJ_ERR_INVALID, "null argument");
  if (!msa->d_chars) return set_error(RNJ_ERR_INVALID, "the alignment was read on the host");
  *d_chars = msa->d_chars;
  if (ld) *ld = (size_t)msa->L;
  return RNJ_OK;
}

int rnj_msa_destroy(rnj_msa *msa) {
  if (msa && msa->d_chars) {
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != msa->device) cudaSetDevice(msa->device);
    cudaFree(msa->d_chars);
    if (prev >= 0 && prev != msa->device) cudaSetDevice(prev);
  }
  delete msa;
  return RNJ_OK;
}

int rnj_write_matrix_text(const char *path, const char *const *names, const float *const *rows,
                          int n, int threads) {
  if (n < 0 || (n > 0 && (!names || !rows))) return set_error(RNJ_ERR_INVALID, "null argument");
  FILE *f = path ? fopen(path, "wb") : stdout;
  if (!f) return set_error(RNJ_ERR_IO, std::string("Could not open the output file \"") + path + "\"");
  fprintf(f, "\t%d\n", n);
  // Rows are formatted in parallel blocks and written in order.
  int T = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
  T = std::max(1, std::min(T, 64));
  const int block = 64;
  std::vector<std::string> text(block);
  for (int r0 = 0; r0 < n; r0 += block) {
    const int rn = std::min(block, n - r0);
    auto work = [&](int k) {
      for (int r = k; r < rn; r += T) {
        std::string &s = text[r];
        s.clear();
        s.append(names[r0 + r] ? names[r0 + r] : "");
        s.push_back('\t');
        char tmp[64];
        for (int j = 0; j < n; ++j) s.append(tmp, format_fixed6(tmp, rows[r0 + r][j]));
        s.push_back('\n');
      }
    };
    std::vector<std::thread> pool;
    const int t = std::min(T, rn);
    for (int k = 1; k < t; ++k) pool.emplace_back(work, k);
    work(0);
    for (auto &th : pool) th.join();
    for (int r = 0; r < rn; ++r) fwrite(text[r].data(), 1, text[r].size(), f);
  }
  if (path) fclose(f);
  else fflush(f);
  return RNJ_OK;
}

}  // extern "C"
