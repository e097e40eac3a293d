/*
 * unifrac_b200.h - C ABI of the B200 Strided State UniFrac engine.
 *
 * The first part of this header is a drop-in for the in-memory and tree
 * entry points of biocore/unifrac-binaries' C API (src/api.hpp).  Types have
 * the same layout, enums the same values, functions the same names,
 * signatures, ownership rules and status codes; each declaration cites the
 * reference declaration it replaces.  Results are allocated by the library
 * with malloc and released only through the matching destroy_*() call.
 *
 * The file-based entry points (one_off, one_off_matrix*, partial,
 * faith_pd_one_off) read BIOM 2.x HDF5 tables with the library's own reader
 * of the HDF5 subset such files use (no HDF5 library) and newick trees;
 * missing or unreadable files give table_missing / tree_missing as the
 * reference, with a message on stderr.
 *
 * The second part (ssu_b200_*) has no counterpart in the reference: in-memory
 * forms of one_off / partial / faith_pd, and a device-resident plan for
 * callers that keep the table on the GPU between calls.
 *
 * Every compute call runs on the current CUDA device (or ACC_DEVICE_NUM when
 * set, as the reference's OpenACC runtime honours it).  Calls are
 * thread-safe: each one owns its stream and device buffers.  No call exits
 * the process; failures come back as a status.
 */
#ifndef UNIFRAC_B200_H
#define UNIFRAC_B200_H

#include <stdint.h>

#ifdef __cplusplus
#define SSU_EXTERN extern "C"
#else
#include <stdbool.h>
#define SSU_EXTERN extern
#endif

/* ------------------------------------------------------------------ types */

/* src/status_enum.hpp:4-6 */
typedef enum compute_status {
    okay = 0, tree_missing, table_missing, table_empty, unknown_method,
    table_and_tree_do_not_overlap, output_error, invalid_method, grouping_missing
} ComputeStatus;
typedef enum io_status {
    read_okay = 0, write_okay, open_error, read_error, magic_incompatible, bad_header, unexpected_end, write_error
} IOStatus;
typedef enum merge_status {
    merge_okay = 0, incomplete_stripe_set, sample_id_consistency, square_mismatch, partials_mismatch, stripes_overlap
} MergeStatus;

/* Condensed (scipy squareform) result, src/api.hpp:40-46. */
typedef struct mat {
    unsigned int n_samples;
    unsigned int cf_size;
    bool is_upper_triangle;
    double *condensed_form;
    char **sample_ids;
} mat_t;

/* Full row-major n x n result, src/api.hpp:54-72.  flags bit 0x1000 marks a
 * matrix backed by an unlinked temp file under mmap_dir (low 12 bits: fd). */
typedef struct mat_full_fp64 {
    uint32_t n_samples;
    uint32_t flags;
    double *matrix;
    char **sample_ids;
} mat_full_fp64_t;

typedef struct mat_full_fp32 {
    uint32_t n_samples;
    uint32_t flags;
    float *matrix;
    char **sample_ids;
} mat_full_fp32_t;

/* Per-sample vector (Faith PD), src/api.hpp:82-86. */
typedef struct results_vec {
    unsigned int n_samples;
    double *values;
    char **sample_ids;
} r_vec;

/* Stripes [stripe_start, stripe_stop) of the distance matrix, each of
 * n_samples values: stripes[s - stripe_start][k] = d(k, (k + s + 1) % n),
 * src/api.hpp:99-107. */
typedef struct partial_mat {
    uint32_t n_samples;
    char **sample_ids;
    double **stripes;
    uint32_t stripe_start;
    uint32_t stripe_stop;
    uint32_t stripe_total;
    bool is_upper_triangle;
} partial_mat_t;

/* src/api.hpp:123-133 */
typedef struct partial_dyn_mat {
    uint32_t n_samples;
    char **sample_ids;
    uint64_t *offsets;
    double **stripes;
    uint32_t stripe_start;
    uint32_t stripe_stop;
    uint32_t stripe_total;
    bool is_upper_triangle;
    char *filename;
} partial_dyn_mat_t;

/* Observation-major CSR table, borrowed for the call: row i (feature
 * obs_ids[i]) spans indptr[i]..indptr[i+1] of indices (sample positions) and
 * data (counts).  src/api.hpp:145-154 */
typedef struct support_biom {
    char **obs_ids;
    char **sample_ids;
    uint32_t *indices;
    uint32_t *indptr;
    double *data;
    int n_obs;
    int n_samples;
    int nnz;
} support_biom_t;

/* Balanced-parentheses tree: structure[i] true for '(' ; the length and name
 * of a node sit at its opening index.  src/api.hpp:163-168 */
typedef struct support_bptree {
    bool *structure;
    double *lengths;
    char **names;
    int n_parens;
} support_bptree_t;

/* Opaque parsed tree, src/api.hpp:173-175. */
typedef struct opaque_bptree {
    int dummy;
} opaque_bptree_t;

/* --------------------------------------------- reference-compatible calls */

/* src/api.hpp:28 - seeds the rarefaction generator. */
SSU_EXTERN void ssu_set_random_seed(unsigned int new_seed);

/* src/api.hpp:188-206 */
SSU_EXTERN IOStatus read_bptree_opaque(const char *tree_filename, opaque_bptree_t **tree_data);
SSU_EXTERN void load_bptree_opaque(const char *newick, opaque_bptree_t **tree_data);
SSU_EXTERN void convert_bptree_opaque(const support_bptree_t *in_tree, opaque_bptree_t **tree_data);
SSU_EXTERN void destroy_bptree_opaque(opaque_bptree_t **tree_data);
/* Number of tips of the tree (the reference returns this too, whatever its comment says). */
SSU_EXTERN int get_bptree_opaque_els(opaque_bptree_t *tree_data);

/* src/api.hpp:196-201 */
SSU_EXTERN void destroy_mat(mat_t **result);
SSU_EXTERN void destroy_mat_full_fp64(mat_full_fp64_t **result);
SSU_EXTERN void destroy_mat_full_fp32(mat_full_fp32_t **result);
SSU_EXTERN void destroy_partial_mat(partial_mat_t **result);
SSU_EXTERN void destroy_partial_dyn_mat(partial_dyn_mat_t **result);
SSU_EXTERN void destroy_results_vec(r_vec **result);

/* In-memory full-matrix UniFrac, fp64 and fp32 results.  src/api.hpp:268-323.
 * The fp64 form rejects fp32 method names (and vice versa) with
 * invalid_method, as src/api.cpp:775-829.  A non-NULL *result is filled in
 * place (the caller pre-allocated it), as src/api.cpp:675-677.
 * subsample_depth > 0 rarefies every sample without replacement first
 * (samples below the depth are dropped); only without-replacement is
 * supported, as the reference. */
SSU_EXTERN ComputeStatus one_off_matrix_inmem_v3(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                                 const char *unifrac_method, bool variance_adjust, double alpha,
                                                 bool bypass_tips, bool normalize_sample_counts, unsigned int n_substeps,
                                                 unsigned int subsample_depth, bool subsample_with_replacement,
                                                 const char *mmap_dir, mat_full_fp64_t **result);
SSU_EXTERN ComputeStatus one_off_matrix_inmem_v2(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                                 const char *unifrac_method, bool variance_adjust, double alpha,
                                                 bool bypass_tips, unsigned int n_substeps, unsigned int subsample_depth,
                                                 bool subsample_with_replacement, const char *mmap_dir,
                                                 mat_full_fp64_t **result);
SSU_EXTERN ComputeStatus one_off_inmem(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                       const char *unifrac_method, bool variance_adjust, double alpha,
                                       bool bypass_tips, unsigned int n_substeps, mat_full_fp64_t **result);
SSU_EXTERN ComputeStatus one_off_matrix_inmem_fp32_v3(const support_biom_t *table_data,
                                                      const support_bptree_t *tree_data, const char *unifrac_method,
                                                      bool variance_adjust, double alpha, bool bypass_tips,
                                                      bool normalize_sample_counts, unsigned int n_substeps,
                                                      unsigned int subsample_depth, bool subsample_with_replacement,
                                                      const char *mmap_dir, mat_full_fp32_t **result);
SSU_EXTERN ComputeStatus one_off_matrix_inmem_fp32_v2(const support_biom_t *table_data,
                                                      const support_bptree_t *tree_data, const char *unifrac_method,
                                                      bool variance_adjust, double alpha, bool bypass_tips,
                                                      unsigned int n_substeps, unsigned int subsample_depth,
                                                      bool subsample_with_replacement, const char *mmap_dir,
                                                      mat_full_fp32_t **result);
SSU_EXTERN ComputeStatus one_off_inmem_fp32(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                            const char *unifrac_method, bool variance_adjust, double alpha,
                                            bool bypass_tips, unsigned int n_substeps, mat_full_fp32_t **result);

/* UniFrac between two dense sample vectors over n_obs features.
 * src/api.hpp:456-478 */
SSU_EXTERN ComputeStatus one_dense_pair_v3t(unsigned int n_obs, const char **obs_ids, const double *sample1,
                                            const double *sample2, const opaque_bptree_t *tree_data,
                                            const char *unifrac_method, bool variance_adjust, double alpha,
                                            bool bypass_tips, bool normalize_sample_counts, double *result);
SSU_EXTERN ComputeStatus one_dense_pair_v3(unsigned int n_obs, const char **obs_ids, const double *sample1,
                                           const double *sample2, const support_bptree_t *tree_data,
                                           const char *unifrac_method, bool variance_adjust, double alpha,
                                           bool bypass_tips, bool normalize_sample_counts, double *result);
SSU_EXTERN ComputeStatus one_dense_pair_v2t(unsigned int n_obs, const char **obs_ids, const double *sample1,
                                            const double *sample2, const opaque_bptree_t *tree_data,
                                            const char *unifrac_method, bool variance_adjust, double alpha,
                                            bool bypass_tips, double *result);
SSU_EXTERN ComputeStatus one_dense_pair_v2(unsigned int n_obs, const char **obs_ids, const double *sample1,
                                           const double *sample2, const support_bptree_t *tree_data,
                                           const char *unifrac_method, bool variance_adjust, double alpha,
                                           bool bypass_tips, double *result);

/* File-based entry points (BIOM-HDF5 table + newick tree).
 * src/api.hpp:228-244, 348-436, 492-493, 805-814.  The table file is read by
 * this library's own BIOM-HDF5 reader (/observation/ids, /sample/ids and the
 * observation-major CSR, as src/biom.cpp:18-255); a missing or unreadable
 * table file is table_missing, a missing or unparsable tree file
 * tree_missing.  The one_off_matrix* calls compute in the method's precision
 * and write the result type's (an fp32 method through one_off_matrix_v3
 * gives fp32 arithmetic in an fp64 matrix), as the reference. */
SSU_EXTERN ComputeStatus one_off_v3(const char *biom_filename, const char *tree_filename, const char *unifrac_method,
                                    bool variance_adjust, double alpha, bool bypass_tips,
                                    bool normalize_sample_counts, unsigned int n_substeps, mat_t **result);
SSU_EXTERN ComputeStatus one_off_wtree_v3(const char *biom_filename, const opaque_bptree_t *tree_data,
                                          const char *unifrac_method, bool variance_adjust, double alpha,
                                          bool bypass_tips, bool normalize_sample_counts, unsigned int n_substeps,
                                          mat_t **result);
SSU_EXTERN ComputeStatus one_off(const char *biom_filename, const char *tree_filename, const char *unifrac_method,
                                 bool variance_adjust, double alpha, bool bypass_tips, unsigned int n_substeps,
                                 mat_t **result);
SSU_EXTERN ComputeStatus one_off_wtree(const char *biom_filename, const opaque_bptree_t *tree_data,
                                       const char *unifrac_method, bool variance_adjust, double alpha,
                                       bool bypass_tips, unsigned int n_substeps, mat_t **result);
SSU_EXTERN ComputeStatus one_off_matrix_v3(const char *biom_filename, const char *tree_filename,
                                           const char *unifrac_method, bool variance_adjust, double alpha,
                                           bool bypass_tips, bool normalize_sample_counts, unsigned int n_substeps,
                                           unsigned int subsample_depth, bool subsample_with_replacement,
                                           const char *mmap_dir, mat_full_fp64_t **result);
SSU_EXTERN ComputeStatus one_off_matrix_fp32_v3(const char *biom_filename, const char *tree_filename,
                                                const char *unifrac_method, bool variance_adjust, double alpha,
                                                bool bypass_tips, bool normalize_sample_counts,
                                                unsigned int n_substeps, unsigned int subsample_depth,
                                                bool subsample_with_replacement, const char *mmap_dir,
                                                mat_full_fp32_t **result);
/* From a pre-parsed tree (read_bptree_opaque / load_bptree_opaque /
 * convert_bptree_opaque): src/api.hpp:355-359. */
SSU_EXTERN ComputeStatus one_off_matrix_v3t(const char *biom_filename, const opaque_bptree_t *tree_data,
                                            const char *unifrac_method, bool variance_adjust, double alpha,
                                            bool bypass_tips, bool normalize_sample_counts, unsigned int n_substeps,
                                            unsigned int subsample_depth, bool subsample_with_replacement,
                                            const char *mmap_dir, mat_full_fp64_t **result);
/* Normalised sample counts: src/api.hpp:362-373. */
SSU_EXTERN ComputeStatus one_off_matrix_v2(const char *biom_filename, const char *tree_filename,
                                           const char *unifrac_method, bool variance_adjust, double alpha,
                                           bool bypass_tips, unsigned int n_substeps, unsigned int subsample_depth,
                                           bool subsample_with_replacement, const char *mmap_dir,
                                           mat_full_fp64_t **result);
SSU_EXTERN ComputeStatus one_off_matrix_v2t(const char *biom_filename, const opaque_bptree_t *tree_data,
                                            const char *unifrac_method, bool variance_adjust, double alpha,
                                            bool bypass_tips, unsigned int n_substeps, unsigned int subsample_depth,
                                            bool subsample_with_replacement, const char *mmap_dir,
                                            mat_full_fp64_t **result);
/* No subsampling: src/api.hpp:375-379. */
SSU_EXTERN ComputeStatus one_off_matrix(const char *biom_filename, const char *tree_filename,
                                        const char *unifrac_method, bool variance_adjust, double alpha,
                                        bool bypass_tips, unsigned int n_substeps, const char *mmap_dir,
                                        mat_full_fp64_t **result);
/* fp32 twins: src/api.hpp:412-436. */
SSU_EXTERN ComputeStatus one_off_matrix_fp32_v3t(const char *biom_filename, const opaque_bptree_t *tree_data,
                                                 const char *unifrac_method, bool variance_adjust, double alpha,
                                                 bool bypass_tips, bool normalize_sample_counts,
                                                 unsigned int n_substeps, unsigned int subsample_depth,
                                                 bool subsample_with_replacement, const char *mmap_dir,
                                                 mat_full_fp32_t **result);
SSU_EXTERN ComputeStatus one_off_matrix_fp32_v2(const char *biom_filename, const char *tree_filename,
                                                const char *unifrac_method, bool variance_adjust, double alpha,
                                                bool bypass_tips, unsigned int n_substeps,
                                                unsigned int subsample_depth, bool subsample_with_replacement,
                                                const char *mmap_dir, mat_full_fp32_t **result);
SSU_EXTERN ComputeStatus one_off_matrix_fp32_v2t(const char *biom_filename, const opaque_bptree_t *tree_data,
                                                 const char *unifrac_method, bool variance_adjust, double alpha,
                                                 bool bypass_tips, unsigned int n_substeps,
                                                 unsigned int subsample_depth, bool subsample_with_replacement,
                                                 const char *mmap_dir, mat_full_fp32_t **result);
SSU_EXTERN ComputeStatus one_off_matrix_fp32(const char *biom_filename, const char *tree_filename,
                                             const char *unifrac_method, bool variance_adjust, double alpha,
                                             bool bypass_tips, unsigned int n_substeps, const char *mmap_dir,
                                             mat_full_fp32_t **result);
SSU_EXTERN ComputeStatus faith_pd_one_off(const char *biom_filename, const char *tree_filename, r_vec **result);
SSU_EXTERN ComputeStatus partial_v3(const char *biom_filename, const char *tree_filename, const char *unifrac_method,
                                    bool variance_adjust, double alpha, bool bypass_tips,
                                    bool normalize_sample_count, unsigned int n_substeps, unsigned int stripe_start,
                                    unsigned int stripe_stop, partial_mat_t **result);
SSU_EXTERN ComputeStatus partial(const char *biom_filename, const char *tree_filename, const char *unifrac_method,
                                 bool variance_adjust, double alpha, bool bypass_tips, unsigned int n_substeps,
                                 unsigned int stripe_start, unsigned int stripe_stop, partial_mat_t **result);

/* Partial results on disk (src/api.hpp:22-23, 816-991): the reference's
 * version-2 file (magic 0x088ABA02, LZ4 blocks of the sample ids and of each
 * stripe), written and read with this library's own LZ4 block codec.
 * Statuses are the reference's; unlike it, a malformed file or an
 * out-of-range stripe index is reported, never fatal.  read_partial_header
 * reads only the header; stripes are then read on demand
 * (read_partial_one_stripe) or by the merges.  validate_partial and the
 * merges need the same samples, stripe total and triangle flag in every
 * partial, no stripe twice and every stripe present (zero partials:
 * incomplete_stripe_set, where the reference exits). */
SSU_EXTERN IOStatus write_partial(const char *filename, const partial_mat_t *result);
SSU_EXTERN IOStatus read_partial(const char *filename, partial_mat_t **result);
SSU_EXTERN IOStatus read_partial_header(const char *input_filename, partial_dyn_mat_t **result_out);
SSU_EXTERN IOStatus read_partial_one_stripe(partial_dyn_mat_t *result, uint32_t stripe_idx);
SSU_EXTERN MergeStatus validate_partial(const partial_dyn_mat_t *const *partial_mats, int n_partials);
SSU_EXTERN MergeStatus merge_partial_to_matrix(partial_dyn_mat_t **partial_mats, int n_partials,
                                               mat_full_fp64_t **result);
SSU_EXTERN MergeStatus merge_partial_to_matrix_fp32(partial_dyn_mat_t **partial_mats, int n_partials,
                                                    mat_full_fp32_t **result);
SSU_EXTERN MergeStatus merge_partial_to_mmap_matrix(partial_dyn_mat_t **partial_mats, int n_partials,
                                                    const char *mmap_dir, mat_full_fp64_t **result);
SSU_EXTERN MergeStatus merge_partial_to_mmap_matrix_fp32(partial_dyn_mat_t **partial_mats, int n_partials,
                                                         const char *mmap_dir, mat_full_fp32_t **result);

/* ------------------------------------------- extensions (no reference twin) */

/* A BIOM-HDF5 table file read into a malloc'ed support_biom_t (ids copied,
 * observation-major CSR), for callers without an HDF5 library; the reference
 * reads the same datasets inside su::biom (src/biom.cpp:18-255) but does not
 * export it.  open_error for a missing file, read_error for a file that is not
 * a readable BIOM-HDF5 table (a message goes to stderr).  Release with
 * ssu_b200_destroy_biom. */
SSU_EXTERN IOStatus ssu_b200_read_biom(const char *biom_filename, support_biom_t **table);
SSU_EXTERN void ssu_b200_destroy_biom(support_biom_t **table);

/* n_subsamples rarefied replicates of a table, drawn on the GPU: samples with
 * a total below `depth` dropped, each kept sample reduced to `depth` counts
 * drawn without replacement (integer-truncated counts, every subset of units
 * equally likely; all units kept when fewer than depth) or with replacement
 * (counts as weights), observations left without counts dropped - the rules
 * of su::skbio_biom_subsampled (src/biom_subsampled.cpp:287-353), whose
 * random stream (libstdc++, thread-count dependent) is not reproduced.
 * Replicate r depends only on seed + r (ssu_set_random_seed) and the
 * sample; the subsample_depth of one_off_matrix_inmem_v3 and of the file
 * calls draws replicate 0.  results[0..n_subsamples) receive malloc'ed tables to release with
 * ssu_b200_destroy_biom.  The ssu_b200_subsample_batch_* calls use the same
 * draws. */
SSU_EXTERN ComputeStatus ssu_b200_rarefy_batch(const support_biom_t *table, unsigned int n_subsamples,
                                               unsigned int depth, bool with_replacement, support_biom_t **results);

/* one_off / partial / faith_pd_one_off over in-memory inputs: the compute
 * paths of the file-based calls above without the file parsing.  Method names,
 * statuses and result layouts are those of the file-based calls.  An
 * out-of-range stripe_stop returns output_error (the reference exits). */
SSU_EXTERN ComputeStatus ssu_b200_one_off_inmem_v3(const support_biom_t *table_data,
                                                   const support_bptree_t *tree_data, const char *unifrac_method,
                                                   bool variance_adjust, double alpha, bool bypass_tips,
                                                   bool normalize_sample_counts, unsigned int n_substeps,
                                                   mat_t **result);
SSU_EXTERN ComputeStatus ssu_b200_partial_inmem_v3(const support_biom_t *table_data,
                                                   const support_bptree_t *tree_data, const char *unifrac_method,
                                                   bool variance_adjust, double alpha, bool bypass_tips,
                                                   bool normalize_sample_counts, unsigned int n_substeps,
                                                   unsigned int stripe_start, unsigned int stripe_stop,
                                                   partial_mat_t **result);
SSU_EXTERN ComputeStatus ssu_b200_faith_pd_inmem(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                                 r_vec **result);

/* Host-side tree helpers used by the tests (no device work): `in_tree`
 * sheared to the tips named in names[0..n_names) (names == NULL keeps every
 * tip) and, when do_collapse, collapsed; written into caller buffers of
 * n_parens slots, *out_n gets its size.  Names are pointers into
 * in_tree->names.  Returns 0 on success. */
SSU_EXTERN int ssu_b200_shear_collapse(const support_bptree_t *in_tree, const char *const *names, int n_names,
                                       int do_collapse, bool *out_structure, double *out_lengths,
                                       const char **out_names, int *out_n);
/* Newick -> BP arrays into caller buffers of `capacity` slots (lengths read
 * through single precision, as the reference's parser).  Names point into a
 * buffer owned by the opaque tree; free it with destroy_bptree_opaque. */
SSU_EXTERN int ssu_b200_tree_arrays(const opaque_bptree_t *tree_data, int capacity, bool *out_structure,
                                    double *out_lengths, const char **out_names, int *out_n);

/* Device-resident plan: the table and tree are prepared and uploaded once;
 * every execute recomputes the full n x n matrix into device memory from the
 * resident inputs.  stream (a cudaStream_t, may be NULL) orders the work. */
typedef struct ssu_b200_plan ssu_b200_plan_t;
SSU_EXTERN ComputeStatus ssu_b200_plan_create(const support_biom_t *table_data, const support_bptree_t *tree_data,
                                              const char *unifrac_method, bool variance_adjust, double alpha,
                                              bool bypass_tips, bool normalize_sample_counts,
                                              ssu_b200_plan_t **plan);
SSU_EXTERN ComputeStatus ssu_b200_plan_execute(ssu_b200_plan_t *plan, void *stream);
/* Device pointer to the n x n result (double for *_fp64 methods, else float). */
SSU_EXTERN const void *ssu_b200_plan_device_result(const ssu_b200_plan_t *plan);
SSU_EXTERN ComputeStatus ssu_b200_plan_copy_result(ssu_b200_plan_t *plan, void *host_out, void *stream);
/* Sum over tables of n(n-1)/2 * embedded branches: the pair-branch updates
 * one execute performs. */
SSU_EXTERN uint64_t ssu_b200_plan_work_units(const ssu_b200_plan_t *plan);
SSU_EXTERN uint32_t ssu_b200_plan_n_samples(const ssu_b200_plan_t *plan);
SSU_EXTERN uint64_t ssu_b200_plan_n_embedded(const ssu_b200_plan_t *plan);
/* Kernel launches one execute issues. */
SSU_EXTERN uint32_t ssu_b200_plan_launches(const ssu_b200_plan_t *plan);
/* Tensor-core int8 operations (2 x multiply-adds; both byte products of
 * each length, chunk padding and the units on the diagonal included) one
 * execute issues on the unweighted tensor-core path; 0 for plans on other
 * kernels. */
SSU_EXTERN uint64_t ssu_b200_plan_tensor_flops(const ssu_b200_plan_t *plan);
/* When enabled, execute brackets each stage with CUDA events on its stream;
 * ssu_b200_plan_stage_ms then reports {embed, pair-kernel, finalize} in ms for
 * the last execute (synchronising the stream), and the pair kernel's
 * algorithmic bytes per launch. */
SSU_EXTERN void ssu_b200_plan_set_timing(ssu_b200_plan_t *plan, int enable);
SSU_EXTERN int ssu_b200_plan_stage_ms(ssu_b200_plan_t *plan, float *embed_ms, float *pair_ms, float *finalize_ms);
SSU_EXTERN void ssu_b200_plan_destroy(ssu_b200_plan_t **plan);

/* Weighted UniFrac (normalized when `normalized` != 0, else unnormalized)
 * for callers that cannot allocate device memory - code running inside a
 * framework that owns all device memory through its own arena, or under a
 * fixed device-memory budget handed out up front.  No counterpart in the
 * reference.  The caller passes device buffers: d_embedding holds
 * n_embedded rows of ld doubles (ld a multiple of 128, >= n_samples), row e
 * the proportions of embedded branch e per sample; d_lengths the n_embedded
 * branch lengths; d_out receives the full n_samples x n_samples fp64 matrix.
 * d_embedding must be 16-byte aligned and d_lengths, d_out 8-byte aligned
 * (output_error otherwise).  The call allocates nothing: its scratch (split-K partial tiles, per-sample
 * weighted sums, tile list) lives in one 32 MiB file-scope device array that
 * every GPU loading the library holds until exit.  n_samples is limited to
 * 100000 and a call whose scratch needs exceed the array returns
 * output_error with a message.  All calls share that array and it keeps the
 * last call's contents (nothing in it needs to start at zero); calls that
 * overlap on the GPU race on it.  The first call on a device resolves the
 * array's address and sets kernel limits, so it should come before any
 * stream capture.  Work is queued on `stream` (a cudaStream_t, may be NULL)
 * and not synchronised. */
SSU_EXTERN ComputeStatus ssu_b200_weighted_pairs_noalloc(const double *d_embedding, const double *d_lengths,
                                                         uint32_t n_embedded, uint32_t n_samples, uint64_t ld,
                                                         int normalized, double *d_out, void *stream);

/* ---- batches: many tables sharing one tree, in one device plan ----------
 *
 * The reference computes several rarefied replicates of a table only inside
 * unifrac_multi_to_file_v2/_v3 (src/api.hpp:565-595), which write them to a
 * file; it has no in-memory batch call.  These entry points take n_tables
 * tables (rarefied replicates, or independent tables of uneven sample
 * counts) that share one tree.  Table t's result equals
 * one_off_matrix_inmem_v3 (or _fp32_v3) on table t alone - the same
 * validation, shear and collapse per table - but the whole batch runs as one
 * plan: tables are embedded together in groups that fit the device, and each
 * group's pair stage is one persistent kernel launch over the tiles of all
 * its tables.  results[0..n_tables) receive malloc'ed matrices to release
 * with destroy_mat_full_fp64 / _fp32; on an error none is left allocated.
 * Environment: UNIFRAC_B200_GROUP_BYTES caps a group's device bytes,
 * UNIFRAC_B200_AUTOTUNE=0 keeps the default tile shapes (batches measure
 * their candidates), UNIFRAC_B200_TUNE_CACHE=<file> keeps tuned choices
 * across processes. */
SSU_EXTERN ComputeStatus ssu_b200_one_off_batch_inmem_v3(const support_biom_t *const *tables, unsigned int n_tables,
                                                         const support_bptree_t *tree_data,
                                                         const char *unifrac_method, bool variance_adjust,
                                                         double alpha, bool bypass_tips,
                                                         bool normalize_sample_counts, mat_full_fp64_t **results);
SSU_EXTERN ComputeStatus ssu_b200_one_off_batch_inmem_fp32_v3(const support_biom_t *const *tables,
                                                              unsigned int n_tables,
                                                              const support_bptree_t *tree_data,
                                                              const char *unifrac_method, bool variance_adjust,
                                                              double alpha, bool bypass_tips,
                                                              bool normalize_sample_counts,
                                                              mat_full_fp32_t **results);
/* The compute part of unifrac_multi_to_file_v3 in memory: n_subsamples
 * replicates of table_data, each rarefied to subsample_depth on the GPU
 * (ssu_b200_rarefy_batch's draws: replicate r under seed s is what
 * one_off_matrix_inmem_v3's subsample_depth draws under seed s + r),
 * computed as one batch; results[r] holds replicate r's matrix over the
 * samples that reached the depth. */
SSU_EXTERN ComputeStatus ssu_b200_subsample_batch_inmem_v3(const support_biom_t *table_data,
                                                           const support_bptree_t *tree_data,
                                                           const char *unifrac_method, bool variance_adjust,
                                                           double alpha, bool bypass_tips,
                                                           bool normalize_sample_counts, unsigned int n_subsamples,
                                                           unsigned int subsample_depth,
                                                           bool subsample_with_replacement,
                                                           mat_full_fp64_t **results);
SSU_EXTERN ComputeStatus ssu_b200_subsample_batch_inmem_fp32_v3(
    const support_biom_t *table_data, const support_bptree_t *tree_data, const char *unifrac_method,
    bool variance_adjust, double alpha, bool bypass_tips, bool normalize_sample_counts, unsigned int n_subsamples,
    unsigned int subsample_depth, bool subsample_with_replacement, mat_full_fp32_t **results);
/* Device-resident batch plan: results of every table, one after the other,
 * in device memory (ssu_b200_plan_table_offset elements in).  group_bytes
 * caps the device bytes of one group's embedding (0: half the free memory);
 * autotune: -1 default, 0 heuristic tile shapes, 1 measured. */
SSU_EXTERN ComputeStatus ssu_b200_batch_plan_create(const support_biom_t *const *tables, unsigned int n_tables,
                                                    const support_bptree_t *tree_data, const char *unifrac_method,
                                                    bool variance_adjust, double alpha, bool bypass_tips,
                                                    bool normalize_sample_counts, uint64_t group_bytes,
                                                    int autotune, ssu_b200_plan_t **plan);
SSU_EXTERN uint32_t ssu_b200_plan_n_tables(const ssu_b200_plan_t *plan);
SSU_EXTERN uint32_t ssu_b200_plan_n_groups(const ssu_b200_plan_t *plan);
SSU_EXTERN uint32_t ssu_b200_plan_table_samples(const ssu_b200_plan_t *plan, uint32_t table);
SSU_EXTERN uint64_t ssu_b200_plan_table_offset(const ssu_b200_plan_t *plan, uint32_t table);
/* Embedded branches of the table's own sheared, collapsed tree. */
SSU_EXTERN uint64_t ssu_b200_plan_table_embedded(const ssu_b200_plan_t *plan, uint32_t table);
/* With enable != 0, the next execute captures the plan's whole launch
 * sequence as one CUDA graph and every later execute launches that graph. */
SSU_EXTERN void ssu_b200_plan_set_graph(ssu_b200_plan_t *plan, int enable);
/* How the pair kernel's tile shape was chosen, and the shape. */
SSU_EXTERN const char *ssu_b200_plan_tuning(const ssu_b200_plan_t *plan);

/* ---- statistics on the distance matrix, on the device ------------------
 *
 * The reference hands these to scikit-bio-binaries (src/skbio_alt.cpp:144-234).
 * Matrices are n_samples x n_samples row-major, in host memory (copied to the
 * device) or device memory (read in place); arithmetic is fp64 throughout.
 * PCoA: the eigenpairs of the Gower-centred -D^2/2 by randomized subspace
 * iteration (Halko, Martinsson and Tropp, 10 extra columns, Rayleigh-Ritz
 * after every multiply, stopped when the wanted Ritz values settle to 1e-12
 * of the largest), the method of scikit-bio's "fsvd" carried to convergence
 * (the reference's fsvd stops after a fixed few steps); each axis has its
 * largest-magnitude entry positive (the reference's signs are arbitrary).
 * Outputs are malloc'ed, released with free(); after a failure (reported on
 * stderr) they are NULL. */

/* src/api.hpp:1008-1010 (C++ linkage there).  eigenvalues[n_dims] descending,
 * samples[n_samples][n_dims] = eigenvector * sqrt(eigenvalue),
 * proportion_explained[n_dims] = eigenvalue / trace of the centred matrix. */
SSU_EXTERN void pcoa(const double *mat, const uint32_t n_samples, const uint32_t n_dims, double **eigenvalues,
                     double **samples, double **proportion_explained);
SSU_EXTERN void pcoa_fp32(const float *mat, const uint32_t n_samples, const uint32_t n_dims, float **eigenvalues,
                          float **samples, float **proportion_explained);
SSU_EXTERN void pcoa_mixed(const double *mat, const uint32_t n_samples, const uint32_t n_dims,
                           float **eigenvalues, float **samples, float **proportion_explained);
/* src/api.hpp:1001-1002, src/api.cpp:2501-2507 (C++ linkage there; the header
 * names the fp32 form find_eigens_fast_p32, the source find_eigens_fast_fp32,
 * which is the one defined).  The n_dims largest eigenpairs of an already
 * centred symmetric matrix: eigenvectors[n_samples][n_dims], unit length.
 * The matrix is not modified. */
SSU_EXTERN void find_eigens_fast(const uint32_t n_samples, const uint32_t n_dims, double *centered,
                                 double **eigenvalues, double **eigenvectors);
SSU_EXTERN void find_eigens_fast_fp32(const uint32_t n_samples, const uint32_t n_dims, float *centered,
                                      float **eigenvalues, float **eigenvectors);
/* src/api.hpp:616-638.  For each of the n_columns grouping columns of the
 * metadata TSV (header line, first field the sample id, tab-separated, as
 * src/tsv.cpp:118-180 reads it): scikit-bio's PERMANOVA pseudo-F over the
 * matrix's upper triangle and its p-value from permanova_perms permutations
 * ((1 + #F_perm >= F) / (1 + perms); NaN with no permutations), drawn from
 * the library seed (ssu_set_random_seed) + column index.  grouping_missing
 * when the file, a column or a sample's line is missing (the reference does
 * not check the first sample; this checks all).  F and p are NaN when there
 * are fewer than 2 groups or as many groups as samples. */
SSU_EXTERN ComputeStatus compute_permanova_fp64(const char *grouping_filename, unsigned int n_columns,
                                                const char **columns, mat_full_fp64_t *result,
                                                unsigned int permanova_perms, double *fstats, double *pvalues);
SSU_EXTERN ComputeStatus compute_permanova_fp32(const char *grouping_filename, unsigned int n_columns,
                                                const char **columns, mat_full_fp32_t *result,
                                                unsigned int permanova_perms, float *fstats, float *pvalues);
/* The grouping column alone: grouping[n_samples] receives group numbers
 * 0, 1, ... in the order their values first appear in the file. */
SSU_EXTERN ComputeStatus ssu_b200_read_grouping(const char *grouping_filename, const char *column,
                                                uint32_t n_samples, const char *const *sample_ids,
                                                uint32_t *grouping, uint32_t *n_groups);
/* PERMANOVA of one grouping given as labels (any values; at most 65535
 * distinct), permutations from the library seed. */
SSU_EXTERN ComputeStatus ssu_b200_permanova_fp64(const double *mat, uint32_t n_samples, const uint32_t *grouping,
                                                 unsigned int permanova_perms, double *fstat, double *pvalue);
SSU_EXTERN ComputeStatus ssu_b200_permanova_fp32(const float *mat, uint32_t n_samples, const uint32_t *grouping,
                                                 unsigned int permanova_perms, float *fstat, float *pvalue);
/* One dataset of an HDF5 file of the subset BIOM files and the reference's
 * outputs use (src/api.cpp:1160-1290: "matrix", "order", "pcoa_eigvals",
 * "pcoa_samples", "pcoa_proportion_explained", "stat_*"): numbers as
 * malloc'ed doubles in row-major order with rank and dims[0..rank) (rank <= 8),
 * strings as a malloc'ed array released with ssu_b200_free_h5_strings. */
SSU_EXTERN IOStatus ssu_b200_read_h5_doubles(const char *filename, const char *dataset, double **values,
                                             uint32_t *rank, uint64_t *dims);
SSU_EXTERN IOStatus ssu_b200_read_h5_strings(const char *filename, const char *dataset, char ***strings,
                                             uint64_t *n);
SSU_EXTERN void ssu_b200_free_h5_strings(char **strings, uint64_t n);

/* Name of the kernel family the plan's pair stage launches (for profiling). */
SSU_EXTERN const char *ssu_b200_plan_pair_kernel(const ssu_b200_plan_t *plan);
/* Library version string. */
SSU_EXTERN const char *ssu_b200_version(void);

#endif /* UNIFRAC_B200_H */
