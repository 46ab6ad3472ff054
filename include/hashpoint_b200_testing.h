/*
 * hashpoint_b200_testing -- test-only C ABI of the B200 HashPoint library.
 *
 * These entry points exist for the library's own tests and are not part of
 * the product library (hashpoint_b200.h): they are compiled, together with the
 * sources they exercise, into a separate shared library,
 * libhashpoint_b200_testing.so, which also exports the product entry points of
 * those sources.  None has a counterpart in the reference.
 */
#ifndef HASHPOINT_B200_TESTING_H
#define HASHPOINT_B200_TESTING_H

#include "hashpoint_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A self-check of the tensor-core operand forms the Aggregator's kernels use.  hp_tc_check_mma runs one
 * tcgen05.mma, d [128, 256] f32 = A [128 x 16] * B [256 x 16]^T in bf16, from
 * device images of shared memory (A: hp_tc_check_image_bytes(0) bytes, B:
 * hp_tc_check_image_bytes(1); 16-byte aligned).  The descriptor of each
 * operand starts a_offset / b_offset bytes into its image, in one of three
 * K-major forms:
 *   HP_TC_PLAIN  no swizzle: 8-row x 16-byte core matrices, K-adjacent ones
 *                128 bytes apart, 8-row groups 256 bytes apart;
 *   HP_TC_SW128  128-byte swizzle: a 128-byte row per matrix row, its 16-byte
 *                chunks permuted by chunk ^ (row % 8), 8-row atoms of 1024 bytes;
 *   HP_TC_SW64   64-byte swizzle: a 64-byte row per matrix row, chunks permuted
 *                by chunk ^ ((row / 2) % 4), 8-row atoms of 512 bytes.
 * Unlike the other entry points it allocates (a 4-byte status word) and
 * synchronises on stream. */
enum { HP_TC_PLAIN = 0, HP_TC_SW128 = 1, HP_TC_SW64 = 2 };
HP_API size_t hp_tc_check_image_bytes(int32_t operand);
HP_API int32_t hp_tc_check_mma(const void* a_image, const void* b_image, int32_t a_form, uint32_t a_offset,
                               int32_t b_form, uint32_t b_offset, float* d, hp_stream_t stream);

/* A test of the Aggregator's bounded waits: hp_aggregator_forward with one
 * weight block (block3.0's extra-input columns) never loaded into the pair
 * kernel's shared memory.  The tensor-core warp's wait for it gives up after
 * wait_limit_us (> 0), the other roles' waits end at once, the kernels return
 * with no copy or MMA in flight, and hp_aggregator_status (on the same
 * workspace and n_samples) reports the failure; the outputs are not valid.
 * The context stays usable. */
HP_API int32_t hp_aggregator_forward_withheld(const void* packed, const float* pc_xyz, const float* pc_rgb,
                                              const float* pc_dir, const float* pc_feat, int32_t feat_dim,
                                              const float* sp_xyz, const uint8_t* valid, const float* rays_d,
                                              int64_t n_samples, int32_t P, const uint8_t* mask_out,
                                              const int32_t* mask_offsets, int64_t n_positions, float* alpha_out,
                                              float* color_out, void* workspace, size_t workspace_bytes,
                                              int32_t wait_limit_us, hp_stream_t stream);

/* A test of the hash-table scan's bounded waits: hp_pts2plane with the scan
 * block that starts withhold_tile-th never publishing its total.  The blocks
 * after it poll it a bounded number of times, give up, count it as empty and
 * flag the failure, which hp_pts2plane_status reports; the outputs are not
 * valid.  The context stays usable. */
HP_API int32_t hp_pts2plane_withheld(const float* xyz, int64_t n_points, const hp_camera* cam, int32_t sort,
                                     int32_t* sorted_point_idx, float* sorted_depth, int32_t* hash_table,
                                     void* workspace, size_t workspace_bytes, int32_t withhold_tile,
                                     hp_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* HASHPOINT_B200_TESTING_H */
