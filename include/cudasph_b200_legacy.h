/*
 * cudasph_b200_legacy.h -- the reference's extern "C" boundary, provided by
 * libcudasph_b200.so so that the reference's unmodified C++ driver
 * (CUDAsph_iterate.cpp, step.cpp, sph_accelerations.cpp, CUDA_calls.cpp,
 * CUDA_gravity.cpp, copy_data_to_from.cpp, memory_alloc_free.cpp,
 * set_device.cpp) links against it.
 *
 * The declarations follow CUDAsph.h:22-48 and radixsort/radixsort.cuh:53-61
 * name for name and argument for argument.  float4 and KeyValuePair are
 * spelled with layout-identical structs here so this header needs no CUDA
 * headers; C linkage makes the symbols the ones the driver imports.
 *
 * Behaviour differences from host_calls.cu (all deliberate):
 *   - the kernels are this library's FP64 kernels; float4 inputs are widened
 *     on the device and results narrowed back;
 *   - the caller's kd_tree buffer is accepted and ignored: the tree is rebuilt
 *     on the device from bodies_pos (the neighbour sets depend only on the
 *     positions and ranges, not on the tree);
 *   - failures print a message and exit(1), as CUDA_SAFE_CALL does
 *     (host_calls.cu:14-22); the native API returns codes instead.
 */
#ifndef CUDASPH_B200_LEGACY_H_
#define CUDASPH_B200_LEGACY_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float x, y, z, w; } sph_legacy_float4;            /* CUDA float4 */
typedef struct { unsigned int key, value; } sph_legacy_kv;          /* KeyValuePair, radixsort.cuh:53-57 */

/* CUDAsph.h:24 / host_calls.cu:30 */
void initCUDA(void);
/* CUDAsph.h:25-28 / host_calls.cu:55-74: cudaMalloc/cudaFree/cudaMemcpy wrappers */
void allocateCUDAarray(void **pos, int n, int device_id);
void deleteCUDAarray(void *pos, int device_id);
void copyArrayToDevice(void *device, const void *host, int n, int device_id);
void copyArrayFromDevice(void *host, const void *device, int n, int device_id);

/* CUDAsph.h:30-31 / host_calls.cu:319-361: direct-N gravity with the spline
 * softening of sph_grav_kernel.cu.  pos = numBodies x {x,y,z,m}, vel =
 * numBodies x {vx,vy,vz,range^2}; accel = {gx,gy,gz,phi}.  p, q ignored. */
void compute_CUDA_gravity(int numBodies, sph_legacy_float4 *accel, float *pos, float *vel, int p, int q,
                          int device_id);
/* CUDAsph.h:32-39 / host_calls.cu:292-317 */
void allocateNBodyArrays(float **pos, int numBodies, int device_id);
void deleteNBodyArrays(float *pos, int device_id);
void zallocateNBodyArrays(float **pos, int numBodies, int device_id);
void zdeleteNBodyArrays(float *pos, int device_id);
void zcopyArrayFromDevice(float *host, const float *device, unsigned int numBodies, int device_id);
void zcopyArrayToDevice(float *device, const float *host, int numBodies, int device_id);

/* CUDAsph.h:41 / host_calls.cu:77-153: solve range = 2h for every body of
 * bodies_hash[0..n_bodies).value with body.w > 0 (n_nodes real bodies);
 * writes bodies_pos[].w and n_ngb[].  Returns the elapsed seconds. */
float host_solve_range(int n_bodies, int n_nodes, float rel_err, sph_legacy_kv *bodies_hash, int *bodies_map,
                       sph_legacy_float4 *bodies_pos, sph_legacy_float4 *bodies_vel, sph_legacy_float4 *kd_tree,
                       int *n_ngb, int device_id);
/* CUDAsph.h:42-43 / host_calls.cu:155-287: find_ngb into the caller's CSR
 * (ngb_offset), density -> hydro_data.x and dots_data, pressure ->
 * hydro_data.y, hydro -> bodies_dots (i-side), hydro_data2.x = v_sig and the
 * per-pair ngb_acc (the caller scatters the j-side, sph_accelerations.cpp:
 * 106-114).  bodies_hash[].key receives the neighbour count (the reference
 * stores the walk length there, dev_find_ngb.cu:84-85). */
float host_sph_accelerations(int n_bodies, int ngb_tot, float av_alpha, float av_beta, sph_legacy_kv *bodies_hash,
                             sph_legacy_kv *bodies_hash_extra, int *bodies_map, int *ngb_list, int *ngb_offset,
                             sph_legacy_float4 *hydro_data, sph_legacy_float4 *dots_data,
                             sph_legacy_float4 *bodies_dots, sph_legacy_float4 *hydro_data2, float *ngb_acc,
                             int device_id);
/* CUDAsph.h:44-47 / host_calls.cu:33-53,364-373 */
int get_device_count(void);
void cuda_set_device(int device_id);
void cuda_set_device0(int device_id);
int cuda_get_device(void);
/* radixsort/radixsort.cuh:59-61: stable sort of `elements` pairs by key
 * (low `bits` bits), in place in pData0; pData1 is scratch. */
void RadixSort(sph_legacy_kv *pData0, sph_legacy_kv *pData1, unsigned int elements, unsigned int bits);

#ifdef __cplusplus
}
#endif

#endif /* CUDASPH_B200_LEGACY_H_ */
