// Host rendezvous of the processes of a run over several GPUs, through files
// in a directory that all of them see: the bootstrap of the process main
// (CHARMING_RDV_DIR; the Python package uses torch.distributed instead).
// Replaces the MPI / NVSHMEM bootstrap of the reference's main
// (src/charming.cu:56-70). Host code only, no CUDA.
//
// Call k of a rank writes <dir>/rdv.<k>.<rank> through a temporary file and
// a rename (a reader never sees part of it), then waits for every rank's
// file of call k and reads them in rank order. A rank writes call k+1 only
// after reading all of call k, so once it has all files of call k+1 every
// rank is done with call k and it removes its own file of call k. The
// directory must be empty when the run starts (one per job).
#pragma once

#include <cerrno>
#include <chrono>
#include <cstdio>
#include <string>
#include <thread>
#include <vector>
#include <sys/stat.h>
#include <unistd.h>

namespace charm_host {

class file_rendezvous {
 public:
  file_rendezvous(std::string dir, int rank, int world, double timeout_s = 300.0)
      : dir_(std::move(dir)), rank_(rank), world_(world), timeout_s_(timeout_s) {}

  // all[world * bytes] <- every rank's `mine`, in rank order. 0, or -1 on an
  // I/O error or when a rank's file did not appear within the timeout.
  int allgather(const void* mine, void* all, size_t bytes) {
    const unsigned long long k = calls_++;
    const std::string tmp = path(k, rank_) + ".tmp";
    FILE* f = fopen(tmp.c_str(), "wb");
    if (!f) return -1;
    const bool wrote = fwrite(mine, 1, bytes, f) == bytes;
    if (fclose(f) != 0 || !wrote || rename(tmp.c_str(), path(k, rank_).c_str()) != 0) return -1;
    const auto t0 = std::chrono::steady_clock::now();
    for (int r = 0; r < world_; r++) {
      unsigned char* dst = static_cast<unsigned char*>(all) + (size_t)r * bytes;
      while (true) {
        FILE* g = fopen(path(k, r).c_str(), "rb");
        if (g) {
          const size_t got = fread(dst, 1, bytes, g);
          fclose(g);
          if (got == bytes) break;
          return -1;  // renamed files are complete: a short one is an error
        }
        if (errno != ENOENT) return -1;
        const double waited =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (waited > timeout_s_) return -1;
        std::this_thread::sleep_for(std::chrono::microseconds(200));
      }
    }
    if (k > 0) unlink(path(k - 1, rank_).c_str());
    return 0;
  }

  int barrier() {
    unsigned char c = 1;
    std::vector<unsigned char> all((size_t)world_);
    return allgather(&c, all.data(), 1);
  }

  // The callbacks of charming_devices (ctx: a file_rendezvous).
  static int allgather_cb(void* ctx, const void* mine, void* all, size_t bytes) {
    return static_cast<file_rendezvous*>(ctx)->allgather(mine, all, bytes);
  }
  static int barrier_cb(void* ctx) { return static_cast<file_rendezvous*>(ctx)->barrier(); }

 private:
  std::string path(unsigned long long k, int r) const {
    return dir_ + "/rdv." + std::to_string(k) + "." + std::to_string(r);
  }
  std::string dir_;
  int rank_, world_;
  double timeout_s_;
  unsigned long long calls_ = 0;
};

}  // namespace charm_host
