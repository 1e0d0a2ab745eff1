/*
 * owl_host.h -- C ABI of the host drivers above libowl: the reference's PRP and LL test loops
 * (Gpu::isPrimePRP, src/Gpu.cpp:1400-1584; Gpu::isPrimeLL, src/Gpu.cpp:1586-1663) with their
 * Gerbicz check, savefiles (src/Saver.cpp, formats "OWL PRP 13" / "OWL LL 13" with CRC32) and
 * result residues, built in C++ on the engine calls of owl.h. Same status codes as owl.h.
 */
#ifndef OWL_HOST_H
#define OWL_HOST_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  uint32_t block_size;    /* Gerbicz block B (reference -block; 1000 by default); divides 10000 */
  uint32_t log_step;      /* res64 log/save step, a multiple of B (reference logStep, 20000) */
  uint32_t check_step;    /* full-check interval, 0 = the reference's baseCheckStep(B) */
  uint32_t stop_after;    /* 0 = run to the end; else stop at the first check point >= start + stop_after */
  uint32_t n_savefiles;   /* savefiles kept (reference -save, 4) */
  uint32_t W, H;          /* FFT shape, 0 = automatic */
  const char* save_dir;   /* directory holding <E>/ (PRP) or ll-<E>/ (LL); NULL = no savefiles */
  uint32_t inject_fault_k;/* test hook: flip one data word once after iteration k (0 = off) */
  int verbose;            /* log lines to stderr */
  uint32_t res_cap;       /* capacity of the checkpoint arrays below (may be 0) */
  uint32_t* res_k;        /* iteration of each logged res64 */
  uint64_t* res_res64;    /* data res64 at that iteration */
  uint32_t* res_n;        /* number of checkpoints written */
  int split;              /* OWL_SPLIT_* flags of include/owl.h (owl_plan_set_split); 0 = FP64 form */
  uint32_t proof_power;   /* PRP: 0 = no proof; else save the 2^p proof residues under save_dir/<E>/proof/
                             and write save_dir/proof/<E>-<p>.proof at the end (reference -proof p) */
  uint32_t column_variant; /* OWL_COL_* of include/owl.h for the column pass; 0 = the shape's default */
} owl_run_opts;

typedef struct {
  int is_prime;           /* PRP: 3^(2^E) == 9 (equals9, src/Gpu.cpp:1036); LL: final value 0 */
  int finished;           /* the test reached its end (vs. stopped by stop_after) */
  uint32_t k;             /* iteration reached */
  uint64_t res64;         /* final: PRP type-1 residue 3^(2^E)/9 (doDiv9, src/Gpu.cpp:1128-1148); LL value */
  uint32_t n_errors;      /* Gerbicz failures (each followed by a reload) */
  char res2048[513];      /* PRP: first 64 words of the type-1 residue, hex, most significant first */
  uint32_t proof_power;   /* power of the proof written (may be lower than asked when resuming without
                             the earlier residues, ProofSet::effectivePower), 0 = none */
  char proof_file[1024];  /* path of the verified proof file, "" = none */
  /* round-off statistics (src/Gpu.cpp:1011-1025, src/Gpu.h:62-81): the per-squaring maximum
     |x - rint(x)| of sampled blocks (the reference's wantROE sampling) fitted by a Gumbel law;
     Z = (0.5 - miu) / beta says how many scale units the 0.5 failure point lies above the typical
     maximum. The reference warns "Danger ROE!" when a log step's Z < 20. */
  uint32_t roe_n;         /* sampled squarings over the whole run */
  float roe_max;          /* their largest round-off */
  float roe_z;            /* Z of the last log step's sample (0 = none) */
  float roe_z_avg;        /* sample-size weighted mean Z over the run (the reference's zAvg) */
  uint32_t n_danger_roe;  /* log steps whose Z fell below 20 */
} owl_run_result;

/* PRP-3 test of 2^E - 1 (src/Gpu.cpp:1400-1584): resumes from save_dir/<E>/ when a savefile exists. */
int owl_prp_run(int device, uint32_t E, const owl_run_opts* opts, owl_run_result* out);
/* LL test of 2^E - 1 (src/Gpu.cpp:1586-1663): resumes from save_dir/ll-<E>/. */
int owl_ll_run(int device, uint32_t E, const owl_run_opts* opts, owl_run_result* out);

/* Savefile I/O on their own, for tools and tests (src/Saver.cpp:16-30, 86-143). check/data hold
   nWords(E) = (E-1)/32+1 words. Return OWL_OK, or OWL_ERR_READ on a bad header or CRC. */
int owl_prp_save(const char* save_dir, uint32_t E, uint32_t k, uint32_t block_size, uint64_t res64,
                 const uint32_t* check, uint32_t n_errors, double elapsed);
int owl_prp_load(const char* save_dir, uint32_t E, uint32_t* k, uint32_t* block_size, uint64_t* res64,
                 uint32_t* check, uint32_t* n_errors, double* elapsed);
int owl_ll_save(const char* save_dir, uint32_t E, uint32_t k, const uint32_t* data, double elapsed);
int owl_ll_load(const char* save_dir, uint32_t E, uint32_t* k, uint32_t* data, double* elapsed);
/* CRC-32 (IEEE 802.3, reflected), the savefile checksum (src/common.cpp crc32) */
uint32_t owl_crc32(const void* data, size_t size);

/* SHA3-256 (FIPS 202) of size bytes, the proof hash (src/sha3.cpp through src/Sha3Hash.h) */
void owl_sha3_256(const void* data, size_t size, uint8_t out[32]);
/* The 2^power iterations whose residues a proof needs, increasing, the last = E
   (ProofSet::ProofSet, src/Proof.cpp:132-185). *n = 2^power; cap may be smaller (then truncated). */
int owl_proof_points(uint32_t E, uint32_t power, uint32_t* points, uint32_t cap, uint32_t* n);
/* Proof::load + Proof::verify (src/Proof.cpp:72-128) on device `device`: *valid = the proof checks
   out, *is_prime = its final residue is 9 (probable prime). OWL_ERR_READ on a malformed file. */
int owl_proof_verify(int device, const char* proof_file, int* valid, int* is_prime);

/* ---- work layer (src/Worktodo.cpp, src/Task.cpp) ---- */
enum { OWL_TASK_PRP = 0, OWL_TASK_LL = 1, OWL_TASK_CERT = 2 }; /* reference Task::Kind PRP, LL, CERT */
typedef struct {
  int kind;               /* OWL_TASK_* */
  uint32_t exponent;
  uint32_t squarings;     /* CERT: squarings of the start value */
  char aid[33];           /* assignment id (32 hex digits) or "" */
  char line[512];         /* the verbatim worktodo line ("" for tasks not from a file) */
} owl_task;

/* One worktodo line (src/Worktodo.cpp:26-87): "PRP=", "PRPDC=" -> PRP; "Test=", "DoubleCheck=" -> LL;
   "Cert=<aid>,1,2,E,-1,squarings" -> CERT. OWL_ERR_ARG for a line the reference ignores. */
int owl_worktodo_parse(const char* line, owl_task* task);
/* The next task for worker `instance`: the best line of <dir>/worktodo-<instance>.txt (the smallest CERT,
   else the smallest exponent), else one moved from <master_dir>/worktodo.txt into the local file
   (src/Worktodo.cpp:90-163). *found = 0 when there is no work. */
int owl_worktodo_get(const char* dir, int instance, const char* master_dir, owl_task* task, int* found);
/* Task::execute (src/Task.cpp:192-242): runs the task with opts (save_dir is set to dir), appends the
   result JSON line to <dir>/results-<instance>.txt (writeResultPRP / LL / CERT, src/Task.cpp:141-190),
   removes the task's line from <dir>/worktodo-<instance>.txt and copies the line to result. */
int owl_task_run(int device, const char* dir, int instance, const owl_task* task, const owl_run_opts* opts,
                 char* result, size_t result_len);
/* Gpu::isCERT (src/Gpu.cpp:1665-1725): `squarings` squarings of the E-bit start value read from
   cert_file ((E-1)/8+1 little-endian bytes), SHA3-256 of the result's bytes. */
int owl_cert_run(int device, uint32_t E, uint32_t squarings, const char* cert_file, uint8_t sha3[32],
                 uint64_t* res64);
/* MD5 of a file as 32 lowercase hex digits (proof::fileHash, src/Proof.cpp:30-37) */
int owl_file_md5(const char* path, char out[33]);

#ifdef __cplusplus
}
#endif
#endif
