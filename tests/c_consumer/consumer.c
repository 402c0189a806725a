/* A C caller of the public header, as a reference-side binding would be:
 * compiled as C11 with warnings as errors and linked against the shipped
 * library.  It uses only host-side entry points (no GPU): the ABI version,
 * status strings, FASTA ingest into the read CSR and the database reader.
 * argv[1]: a FASTA file; argv[2]: a database path prefix.  Prints one line
 * per check; exits non-zero on the first failure. */
#include <stdio.h>
#include <string.h>

#include "gkc/gkc.h"

#define CHECK(cond, what)                  \
  do {                                     \
    if (!(cond)) {                         \
      fprintf(stderr, "FAIL %s\n", what);  \
      return 1;                            \
    }                                      \
    printf("ok %s\n", what);               \
  } while (0)

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  CHECK(gkc_abi_version() == GKC_ABI_VERSION, "abi version");
  CHECK(strcmp(gkc_status_string(GKC_ERR_BUDGET), "HBM budget exceeded") == 0, "status string");

  char *reads = NULL;
  uint64_t *offs = NULL, n_reads = 0;
  /* the reference's rule: the line after each header */
  CHECK(gkc_fastx_load(argv[1], 2, 0, &reads, &offs, &n_reads) == GKC_OK && n_reads == 2 && offs[2] == 16 &&
            memcmp(reads, "ACGTACGTGGGGCCCC", 16) == 0,
        "fastx load");
  gkc_fastx_free(reads, offs, 0);
  /* the lines of a record joined */
  CHECK(gkc_fastx_load_ex(argv[1], 2, 0, GKC_FASTX_JOIN_LINES, &reads, &offs, &n_reads) == GKC_OK, "fastx joined");
  CHECK(n_reads == 2 && offs[0] == 0 && offs[1] == 8 && offs[2] == 20, "fastx offsets");
  CHECK(memcmp(reads, "ACGTACGTGGGGCCCCAAAA", 20) == 0, "fastx bytes");
  gkc_fastx_free(reads, offs, 0);

  gkc_db *db = NULL;
  CHECK(gkc_db_open(argv[2], &db) == GKC_OK, "db open");
  gkc_db_info info;
  CHECK(gkc_db_get_info(db, &info) == GKC_OK && info.k == 31 && info.n_kmers == 3, "db info");
  uint64_t keys[4] = {5, 77, 1ull << 40, 6};
  uint32_t counts[4];
  CHECK(gkc_db_lookup(db, keys, 4, counts) == GKC_OK, "db lookup");
  CHECK(counts[0] == 2 && counts[1] == 9 && counts[2] == 300 && counts[3] == 0, "db counts");
  uint64_t k2[3];
  uint32_t c2[3];
  CHECK(gkc_db_read(db, 0, 3, k2, c2) == GKC_OK && k2[0] == 5 && k2[2] == (1ull << 40) && c2[1] == 9, "db read");
  gkc_db_close(db);
  CHECK(gkc_db_open("/nonexistent/db", &db) == GKC_ERR_NOT_FOUND, "db missing");
  return 0;
}
