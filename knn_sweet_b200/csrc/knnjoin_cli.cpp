// knnjoin_cli.cpp -- drop-in for the reference's `knnjoin` command line
// (src/knnjoin.cu:983-1172), running the join through libknnsweet.
//
//   knnjoin query_nb source_nb dim qrep_nb srep_nb K query_file source_file
//
// Inputs as in the reference's pointSetup (include/common8.h:92-135):
// whitespace-separated floats read row-major, query_nb*dim (source_nb*dim)
// values from the start of the file whatever its line structure (parsed on
// all host threads, with the serial reader's result), a raw float32 file
// named *.f32, or the word `random`: after srand(2015), each value is rand()%10 + (float)rand()/RAND_MAX
// (queries first, then sources, from one sequence; the left rand() call is
// evaluated first, as the reference's host compiler does).
//
// Output lines kept from the reference: "total time %f" (seconds; here the
// device time of the whole join, representative draw included), "Total %d"
// (exact distance evaluations) and the K lines "i,k %d %d  %d %f" for query
// 100 (knnjoin.cu:1136-1145).  With KNNJOIN_DUMP=<path> the full result is
// written there as the reference's IndexDist array {int32 index; float dist}
// (query_nb*K records).  Errors go to stderr with exit status 1.
#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "knnsweet.h"
#include "../csrc/glibc_rand.h"

namespace {

bool is_space(char c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

// The serial reader: floats from p on as successive fscanf("%f") calls
// would read them (strtof skips leading whitespace, a token such as "1.5-2"
// yields two values), into out[i ..) until `count` or the first text that is
// not a number.  Returns the new count.
int64_t parse_serial(const char *p, float *out, int64_t i, int64_t count) {
  while (i < count) {
    char *end = nullptr;
    errno = 0;
    const float v = strtof(p, &end);
    if (end == p) break;  // not a number (or end of input)
    out[i++] = v;
    p = end;
  }
  return i;
}

// Reads `count` floats from `path` with the serial reader's result, in
// parallel: the text is cut into chunks at whitespace (no token straddles
// two), the tokens of each chunk are counted, and each chunk is parsed into
// its place.  A chunk holding a token that is not exactly one number (a
// partial parse or a failure) hands the rest of the input, from that chunk
// on, to the serial reader.  Returns the number read; slots past it stay 0.
int64_t read_text_floats(std::vector<char> &buf, float *out, int64_t count) {
  const int64_t size = (int64_t)buf.size() - 1;  // buf ends with '\0'
  const char *t = buf.data();
  const int64_t min_chunk = 1 << 16;
  int nch = (int)std::min<int64_t>(256, std::max<int64_t>(1, size / min_chunk));
  std::vector<int64_t> cb(nch + 1);
  cb[0] = 0;
  for (int c = 1; c < nch; c++) {
    int64_t x = std::max(cb[c - 1], size * c / nch);
    while (x < size && !is_space(t[x])) x++;  // a chunk starts at whitespace
    cb[c] = x;
  }
  cb[nch] = size;
  std::vector<int64_t> ntok(nch + 1, 0);
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < nch; c++) {
    int64_t n = 0;
    bool in_tok = false;
    for (int64_t x = cb[c]; x < cb[c + 1]; x++) {
      const bool sp = is_space(t[x]);
      n += (!sp && !in_tok);
      in_tok = !sp;
    }
    ntok[c + 1] = n;
  }
  for (int c = 0; c < nch; c++) ntok[c + 1] += ntok[c];  // first token index per chunk
  std::vector<char> irregular(nch, 0);
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < nch; c++) {
    int64_t i = ntok[c];
    if (i >= count) continue;
    const char *p = t + cb[c], *e = t + cb[c + 1];
    while (i < count) {
      while (p < e && is_space(*p)) p++;
      if (p == e) break;
      const char *tok_end = p;
      while (tok_end < e && !is_space(*tok_end)) tok_end++;
      char *end = nullptr;
      const float v = strtof(p, &end);
      if (end != tok_end) {  // not a whole number: the serial reader decides
        irregular[c] = 1;
        break;
      }
      out[i++] = v;
      p = tok_end;
    }
  }
  int first_bad = -1;
  for (int c = 0; c < nch && first_bad < 0; c++)
    if (irregular[c] && ntok[c] < count) first_bad = c;
  int64_t got;
  if (first_bad < 0) {
    got = std::min<int64_t>(count, ntok[nch]);
  } else {
    got = parse_serial(t + cb[first_bad], out, ntok[first_bad], count);
    std::fill(out + got, out + count, 0.0f);  // later chunks wrote past the stop
  }
  return got;
}

// Reads `count` floats from `path`: raw little-endian float32 when the name
// ends in ".f32", else whitespace-separated text as the reference's
// fscanf("%f") loop reads it (tokens separated by any whitespace, CRLF
// included; stops at the first token that is not a number).  Returns the
// number read.
int64_t read_floats(const char *path, float *out, int64_t count, bool *open_ok) {
  FILE *f = fopen(path, "rb");
  *open_ok = f != nullptr;
  if (!f) return 0;
  std::vector<char> buf;
  if (fseek(f, 0, SEEK_END) == 0) {
    const long sz = ftell(f);
    if (sz > 0 && fseek(f, 0, SEEK_SET) == 0) {
      buf.resize((size_t)sz);
      buf.resize(fread(buf.data(), 1, (size_t)sz, f));
    }
  }
  if (buf.empty()) {  // size unknown (a pipe): read to the end
    rewind(f);
    char tmp[1 << 16];
    size_t got;
    while ((got = fread(tmp, 1, sizeof tmp, f)) > 0) buf.insert(buf.end(), tmp, tmp + got);
  }
  fclose(f);
  const size_t len = std::strlen(path);
  if (len >= 4 && std::strcmp(path + len - 4, ".f32") == 0) {
    const int64_t have = std::min<int64_t>(count, (int64_t)(buf.size() / sizeof(float)));
    std::memcpy(out, buf.data(), (size_t)have * sizeof(float));
    return have;
  }
  buf.push_back('\0');
  return read_text_floats(buf, out, count);
}

void fill_random(knnsweet::GlibcRand &g, float *out, int64_t count) {
  for (int64_t i = 0; i < count; i++) {
    const int a = g.next();  // rand() % 10, evaluated first
    const int b = g.next();  // (float)rand() / RAND_MAX
    out[i] = (float)(a % 10) + (float)b / (float)2147483647;
  }
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 9) {
    std::printf("usage: ./exe query_nb source_nb dimension qrep_nb srep_nb k input1 input2\n");
    return 1;
  }
  const int64_t query_nb = atoll(argv[1]);
  const int64_t source_nb = atoll(argv[2]);
  const int dim = atoi(argv[3]);
  const int qrep_nb = atoi(argv[4]);
  const int srep_nb = atoi(argv[5]);
  const int K = atoi(argv[6]);
  const char *query_data = argv[7];
  const char *source_data = argv[8];
  if (query_nb < 0 || source_nb < 0 || dim <= 0 || K <= 0 || qrep_nb < 0 || srep_nb < 0) {
    std::fprintf(stderr, "knnjoin: bad arguments\n");
    return 1;
  }
  std::vector<float> queries((size_t)(query_nb * dim)), sources((size_t)(source_nb * dim));

  knnsweet::GlibcRand g(2015);  // srand(2015) once, common8.h:94
  if (std::strcmp(query_data, "random") == 0) {
    std::printf("query data random\n");
    fill_random(g, queries.data(), (int64_t)queries.size());
  } else {
    bool ok = false;
    int64_t got = read_floats(query_data, queries.data(), (int64_t)queries.size(), &ok);
    if (!ok) {
      std::printf("error opening query files\n");
      return 1;
    }
    if (got < (int64_t)queries.size()) std::printf("error reading\n");
  }
  if (std::strcmp(source_data, "random") == 0) {
    std::printf("source data random\n");
    fill_random(g, sources.data(), (int64_t)sources.size());
  } else {
    bool ok = false;
    read_floats(source_data, sources.data(), (int64_t)sources.size(), &ok);
    if (!ok) {
      std::printf("error opening query files\n");  // the reference's wording
      return 1;
    }
  }

  // KNNJOIN_DUMP_INPUT=<path>: write the parsed queries then sources (float32)
  // and stop before the join (checks the reader without a GPU)
  if (const char *dump = std::getenv("KNNJOIN_DUMP_INPUT")) {
    FILE *f = fopen(dump, "wb");
    bool ok = f && fwrite(queries.data(), sizeof(float), queries.size(), f) == queries.size() &&
              fwrite(sources.data(), sizeof(float), sources.size(), f) == sources.size();
    if (f) fclose(f);
    if (!ok) {
      std::fprintf(stderr, "knnjoin: cannot write %s\n", dump);
      return 1;
    }
    return 0;
  }

  knn_options opt;
  knn_default_options(&opt);
  opt.qreps = qrep_nb;
  opt.sreps = srep_nb;
  std::vector<int32_t> idx((size_t)(query_nb * K));
  std::vector<float> dist((size_t)(query_nb * K));
  knn_stats st;
  // the same file twice is a self-join (run_sample.sh:1)
  const bool self = std::strcmp(query_data, source_data) == 0 &&
                    std::strcmp(query_data, "random") != 0 && query_nb == source_nb;
  const float *src = self ? queries.data() : sources.data();
  int rc = knn_join(queries.data(), query_nb, src, source_nb, dim, K, idx.data(),
                    dist.data(), &opt, &st);
  if (rc != KNN_OK) {
    std::fprintf(stderr, "knnjoin: %s\n", knn_last_error());
    return 1;
  }
  std::printf("total time %f\n", st.ms_total / 1000.0);
  std::printf("Total %lld\n", (long long)st.dist_evals);
  const int64_t i = 100;
  if (i < query_nb)
    for (int j = 0; j < K; j++)
      std::printf("i,k %d %d  %d %f\n", (int)i, j, idx[(size_t)(i * K + j)],
                  dist[(size_t)(i * K + j)]);
  if (const char *dump = std::getenv("KNNJOIN_DUMP")) {
    std::vector<uint32_t> rec((size_t)(2 * query_nb * K));
    knn_pack_indexdist(idx.data(), dist.data(), query_nb * K, rec.data());
    FILE *f = fopen(dump, "wb");
    if (!f || fwrite(rec.data(), sizeof(uint32_t), rec.size(), f) != rec.size()) {
      std::fprintf(stderr, "knnjoin: cannot write %s\n", dump);
      if (f) fclose(f);
      return 1;
    }
    fclose(f);
  }
  return 0;
}
