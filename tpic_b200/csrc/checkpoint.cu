// Checkpoints and restart (host code): the state's E (nodes), B (cells) and
// particle records in their stored types, with the cycle, in one piece file
// per checkpoint directory, as TPIC's checkpoint engine lays out its
// directories (src/io/checkpoint.cpp:34-130,362-470; docs/user/output.md,
// "Checkpoints and restart"): `checkpoint_tNNNNNN_n000001/` with the piece
// `checkpoint_tNNNNNN_r000000.tpcb`, written under a hidden name, flushed and
// renamed, older complete checkpoints removed afterwards. The file format is
// this library's: the magic "TPICB200", the tpicb200_checkpoint_info header,
// the arrays in a fixed order and an FNV-1a 64-bit checksum of the arrays.
#include "kernels.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <string>
#include <system_error>
#include <vector>

#include <fcntl.h>
#include <unistd.h>

namespace fs = std::filesystem;
using namespace tpicb200;

namespace {

constexpr char kMagic[8] = {'T', 'P', 'I', 'C', 'B', '2', '0', '0'};
constexpr int kVersion = 1;
constexpr size_t kChunk = size_t(64) << 20;  // host staging per copy

struct Fnv1a {
  uint64_t h = 1469598103934665603ULL;
  void add(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ULL;
  }
};

std::string checkpoint_dir(int cycle) {
  char name[64];
  std::snprintf(name, sizeof name, "checkpoint_t%06d_n000001", cycle);
  return name;
}
std::string piece_file(int cycle) {
  char name[64];
  std::snprintf(name, sizeof name, "checkpoint_t%06d_r000000.tpcb", cycle);
  return name;
}
// The cycle of a checkpoint directory name of this layout (one rank), or -1.
int parse_dir(const std::string& name) {
  int cycle = -1, ranks = -1, used = 0;
  if (std::sscanf(name.c_str(), "checkpoint_t%d_n%d%n", &cycle, &ranks, &used) != 2) return -1;
  if (size_t(used) != name.size() || cycle < 0 || ranks != 1 || name != checkpoint_dir(cycle)) return -1;
  return cycle;
}

// The arrays of a checkpoint in file order: device pointer and bytes.
struct Section {
  void* device;
  size_t bytes;
};
std::vector<Section> sections(const Geom& g, const tpicb200_checkpoint_info& info, const tpicb200_state* st) {
  const size_t fs_ = info.precision == TPICB200_PRECISION_DOUBLE ? 8 : 4;
  std::vector<Section> out;
  out.push_back({st ? st->e : nullptr, size_t(3) * size_t(g.nodes) * fs_});
  out.push_back({st ? st->b_cell : nullptr, size_t(3) * size_t(g.cells) * fs_});
  for (int s = 0; s < info.ns; ++s) {
    const size_t n = info.count[s];
    const tpicb200_particles* p = st ? &st->slot[s][st->current[s]] : nullptr;
    out.push_back({p ? p->rx : nullptr, 8 * n});
    out.push_back({p ? p->ry : nullptr, 8 * n});
    out.push_back({p ? p->rz : nullptr, 8 * n});
    out.push_back({p ? p->u : nullptr, fs_ * n});
    out.push_back({p ? p->v : nullptr, fs_ * n});
    out.push_back({p ? p->w : nullptr, fs_ * n});
    out.push_back({p ? (void*)p->q : nullptr, 8 * n});
    out.push_back({p ? (void*)p->cell : nullptr, 4 * n});
    if (info.has_id[s]) out.push_back({p ? (void*)p->id : nullptr, 8 * n});
  }
  return out;
}

size_t payload_bytes(const std::vector<Section>& secs) {
  size_t total = 0;
  for (const auto& s : secs) total += s.bytes;
  return total;
}

bool grids_equal(const tpicb200_grid& a, const tpicb200_grid& b) {
  return a.nx == b.nx && a.ny == b.ny && a.nz == b.nz && a.lx == b.lx && a.ly == b.ly && a.lz == b.lz;
}

struct File {
  std::FILE* f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

// Reads and validates the magic and header; `size` receives the file size.
int read_header(std::FILE* f, tpicb200_checkpoint_info* info, long long* size, const std::string& path) {
  char magic[8];
  if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kMagic, 8) != 0)
    return report_error(TPICB200_INVALID_DATA, path + ": not a checkpoint piece of this library");
  if (std::fread(info, sizeof *info, 1, f) != 1)
    return report_error(TPICB200_INVALID_DATA, path + ": truncated checkpoint header");
  if (info->version != kVersion || info->ns < 1 || info->ns > TPICB200_MAX_SPECIES ||
      (info->precision != TPICB200_PRECISION_DOUBLE && info->precision != TPICB200_PRECISION_MIXED) ||
      info->grid.nx < 1 || info->grid.ny < 1 || info->grid.nz < 1)
    return report_error(TPICB200_INVALID_DATA, path + ": unsupported or corrupt checkpoint header");
  std::error_code ec;
  *size = (long long)fs::file_size(path, ec);
  if (ec) return report_error(TPICB200_INVALID_DATA, path + ": " + ec.message());
  const Geom g = make_geom(info->grid);
  const long long expected = 8 + (long long)sizeof *info + (long long)payload_bytes(sections(g, *info, nullptr)) + 8;
  if (*size != expected) return report_error(TPICB200_INVALID_DATA, path + ": incomplete checkpoint piece");
  return TPICB200_SUCCESS;
}

}  // namespace

extern "C" {

int tpicb200_checkpoint_write(tpicb200_context* ctx, tpicb200_state* st, const char* directory, int cycle,
                              tpicb200_stream stream) {
  if (!directory || cycle < 0) return report_error(TPICB200_INVALID_ARGUMENT, "checkpoint needs a directory and a cycle");
  if (int r = context_check_state(ctx, st)) return r;
  if (int r = tpicb200_materialize(ctx, st, stream)) return r;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaStreamSynchronize(s) != cudaSuccess) return report_error(TPICB200_BACKEND_FAILURE, "checkpoint: stream failed");
  const Geom& g = context_geom(ctx);
  const tpicb200_options& opt = context_options(ctx);
  tpicb200_checkpoint_info info{};
  info.version = kVersion;
  info.precision = opt.precision;
  info.cycle = cycle;
  info.ns = st->ns;
  info.grid = context_grid(ctx);
  info.dt = opt.dt;
  info.c = opt.c;
  for (int sp = 0; sp < st->ns; ++sp) {
    info.qom[sp] = st->qom[sp];
    info.count[sp] = st->slot[sp][st->current[sp]].count;
    info.has_id[sp] = st->slot[sp][st->current[sp]].id ? 1 : 0;
  }
  std::error_code ec;
  const fs::path dir = fs::path(directory) / checkpoint_dir(cycle);
  fs::create_directories(dir, ec);
  if (ec) return report_error(TPICB200_BACKEND_FAILURE, dir.string() + ": " + ec.message());
  const fs::path final_path = dir / piece_file(cycle);
  const fs::path partial = dir / ("." + piece_file(cycle) + ".partial");
  {
    File out;
    out.f = std::fopen(partial.c_str(), "wb");
    if (!out.f) return report_error(TPICB200_BACKEND_FAILURE, partial.string() + ": cannot create");
    bool ok = std::fwrite(kMagic, 1, 8, out.f) == 8 && std::fwrite(&info, sizeof info, 1, out.f) == 1;
    Fnv1a sum;
    std::vector<unsigned char> stage(kChunk);
    for (const Section& sec : sections(g, info, st)) {
      for (size_t done = 0; ok && done < sec.bytes; done += kChunk) {
        const size_t n = std::min(kChunk, sec.bytes - done);
        if (cudaMemcpyAsync(stage.data(), static_cast<const char*>(sec.device) + done, n, cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
          return report_error(TPICB200_BACKEND_FAILURE, "checkpoint: device copy failed");
        sum.add(stage.data(), n);
        ok = std::fwrite(stage.data(), 1, n, out.f) == n;
      }
    }
    ok = ok && std::fwrite(&sum.h, sizeof sum.h, 1, out.f) == 1;
    ok = ok && std::fflush(out.f) == 0 && ::fsync(::fileno(out.f)) == 0;
    if (!ok) return report_error(TPICB200_BACKEND_FAILURE, partial.string() + ": write failed");
  }
  fs::rename(partial, final_path, ec);
  if (ec) return report_error(TPICB200_BACKEND_FAILURE, final_path.string() + ": " + ec.message());
  if (int fd = ::open(dir.c_str(), O_RDONLY); fd >= 0) {
    ::fsync(fd);
    ::close(fd);
  }
  // The disk keeps the newest complete checkpoint: older ones go.
  for (const auto& entry : fs::directory_iterator(fs::path(directory), ec)) {
    const int other = parse_dir(entry.path().filename().string());
    if (other >= 0 && other < cycle) fs::remove_all(entry.path(), ec);
  }
  return TPICB200_SUCCESS;
}

int tpicb200_checkpoint_find(const char* directory, char* path, size_t size) {
  if (!directory || !path || size == 0) return report_error(TPICB200_INVALID_ARGUMENT, "invalid checkpoint query");
  std::error_code ec;
  int best = -1;
  fs::path found;
  for (const auto& entry : fs::directory_iterator(fs::path(directory), ec)) {
    const int cycle = parse_dir(entry.path().filename().string());
    if (cycle <= best) continue;
    const fs::path piece = entry.path() / piece_file(cycle);
    if (fs::is_regular_file(piece, ec)) {
      best = cycle;
      found = piece;
    }
  }
  if (best < 0) return report_error(TPICB200_INVALID_ARGUMENT, std::string(directory) + ": no complete checkpoint");
  const std::string text = found.string();
  if (text.size() + 1 > size) return report_error(TPICB200_INVALID_ARGUMENT, "checkpoint path does not fit");
  std::memcpy(path, text.c_str(), text.size() + 1);
  return TPICB200_SUCCESS;
}

int tpicb200_checkpoint_info_read(const char* path, tpicb200_checkpoint_info* info) {
  if (!path || !info) return report_error(TPICB200_INVALID_ARGUMENT, "invalid checkpoint query");
  File in;
  in.f = std::fopen(path, "rb");
  if (!in.f) return report_error(TPICB200_INVALID_DATA, std::string(path) + ": cannot open");
  long long size = 0;
  return read_header(in.f, info, &size, path);
}

int tpicb200_checkpoint_read(tpicb200_context* ctx, tpicb200_state* st, const char* path,
                             tpicb200_checkpoint_info* info_out, tpicb200_stream stream) {
  if (!path) return report_error(TPICB200_INVALID_ARGUMENT, "checkpoint needs a path");
  if (int r = context_check_state(ctx, st)) return r;
  const Geom& g = context_geom(ctx);
  const tpicb200_options& opt = context_options(ctx);
  File in;
  in.f = std::fopen(path, "rb");
  if (!in.f) return report_error(TPICB200_INVALID_DATA, std::string(path) + ": cannot open");
  tpicb200_checkpoint_info info{};
  long long size = 0;
  if (int r = read_header(in.f, &info, &size, path)) return r;
  // The run must be the checkpoint's (prepare_restart, src/io/checkpoint.cpp:388-404).
  if (!grids_equal(info.grid, context_grid(ctx)) || info.dt != opt.dt || info.c != opt.c)
    return report_error(TPICB200_INVALID_ARGUMENT, std::string(path) + ": mesh, dt or c differ from the checkpoint's");
  if (info.precision != opt.precision)
    return report_error(TPICB200_INVALID_ARGUMENT, std::string(path) + ": storage precision differs from the checkpoint's");
  if (info.ns != st->ns) return report_error(TPICB200_INVALID_ARGUMENT, std::string(path) + ": species count differs");
  for (int sp = 0; sp < st->ns; ++sp) {
    if (info.qom[sp] != st->qom[sp]) return report_error(TPICB200_INVALID_ARGUMENT, std::string(path) + ": q/m differs");
    if (info.count[sp] > opt.max_particles)
      return report_error(TPICB200_CAPACITY_EXCEEDED, std::string(path) + ": more records than the context holds");
    if (info.has_id[sp] && !st->slot[sp][st->current[sp]].id)
      return report_error(TPICB200_INVALID_ARGUMENT, std::string(path) + ": the checkpoint holds ids, the state none");
  }
  // The checksum first: nothing is written from a corrupt piece.
  std::vector<unsigned char> stage(kChunk);
  const long long header = 8 + (long long)sizeof info;
  const size_t payload = size_t(size - header - 8);
  Fnv1a sum;
  for (size_t done = 0; done < payload; done += kChunk) {
    const size_t n = std::min(kChunk, payload - done);
    if (std::fread(stage.data(), 1, n, in.f) != n)
      return report_error(TPICB200_INVALID_DATA, std::string(path) + ": read failed");
    sum.add(stage.data(), n);
  }
  uint64_t stored = 0;
  if (std::fread(&stored, sizeof stored, 1, in.f) != 1 || stored != sum.h)
    return report_error(TPICB200_INVALID_DATA, std::string(path) + ": checksum mismatch");
  for (int sp = 0; sp < st->ns; ++sp) {
    for (int k = 0; k < 2; ++k) st->slot[sp][k].count = info.count[sp];
    st->ranked[sp] = 0;
  }
  if (std::fseek(in.f, header, SEEK_SET) != 0)
    return report_error(TPICB200_INVALID_DATA, std::string(path) + ": seek failed");
  cudaStream_t s = (cudaStream_t)stream;
  for (const Section& sec : sections(g, info, st)) {
    for (size_t done = 0; done < sec.bytes; done += kChunk) {
      const size_t n = std::min(kChunk, sec.bytes - done);
      if (std::fread(stage.data(), 1, n, in.f) != n)
        return report_error(TPICB200_INVALID_DATA, std::string(path) + ": read failed");
      if (cudaMemcpyAsync(static_cast<char*>(sec.device) + done, stage.data(), n, cudaMemcpyHostToDevice, s) !=
              cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess)
        return report_error(TPICB200_BACKEND_FAILURE, "checkpoint: device copy failed");
    }
  }
  if (info_out) *info_out = info;
  return TPICB200_SUCCESS;
}

}  // extern "C"
