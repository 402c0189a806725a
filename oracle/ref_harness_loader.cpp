// Reference harness, read loader.  TEST INFRASTRUCTURE (oracle/_ref).
// Compiles the reference's ReadLoader (read_loader.hpp) from its sources and
// runs it through its own driver, ReadLoader::work_while_loading (the loader
// on its threads, batches handed to a callback as they are loaded), and
// returns the reads the callbacks receive, in order, as a CSR.  (load_file
// alone stalls once more than two batches wait unconsumed.)
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "utilities.hpp"  // PAR, which read_loader.hpp's driver functions name
#include "read_loader.hpp"

extern "C" int ref_load_reads(const char *path, int n_threads, uint64_t buffer_size, uint64_t *n_reads,
                              char **reads, uint64_t **offs) {
  std::vector<char> bytes;
  std::vector<uint64_t> o(1, 0);
  ReadLoader::work_while_loading(
      [&](vector<ReadPtr> &batch) {
        for (const ReadPtr &r : batch) {
          bytes.insert(bytes.end(), r.read, r.read + r.len);
          o.push_back(bytes.size());
        }
      },
      n_threads < 1 ? 1 : n_threads, std::string(path), 2000, false,
      buffer_size ? buffer_size : 20 * ReadLoader::MB);
  *reads = (char *)malloc(bytes.size() + 1);
  *offs = (uint64_t *)malloc(8 * o.size());
  if (!bytes.empty()) memcpy(*reads, bytes.data(), bytes.size());
  memcpy(*offs, o.data(), 8 * o.size());
  *n_reads = o.size() - 1;
  return 0;
}

extern "C" void ref_free_reads(char *reads, uint64_t *offs) {
  free(reads);
  free(offs);
}
