/*
 * supra_b200 — C ABI of the B200 receive-processing path (DAS, MV, envelope/IQ, log compression,
 * scan conversion) that stands in for SUPRA's receive nodes.
 *
 * Conventions
 *  - Every entry point returns an int status: SB_OK (0) or a negative SB_ERR_* code. The message of
 *    the last failure on the calling thread is returned by sb_last_error(). No C++ exception crosses
 *    this boundary.
 *  - All data pointers passed to *_run functions are DEVICE pointers owned by the caller; nothing is
 *    synchronised with the host. Work is enqueued on the caller's stream (a cudaStream_t passed as
 *    sb_stream; NULL is the legacy default stream). This mirrors SUPRA, whose nodes launch on the
 *    stream of the input container and never synchronise (SupraLib/Container.h:104-108).
 *  - Plans own device copies of geometry, filters and look-up tables. A plan is not thread safe:
 *    one plan per node, as SUPRA serialises each node body under the node mutex
 *    (SupraLib/AbstractNode.h:119-132).
 *  - Layouts follow the reference: raw channel data [tx][channel][sample] (Beamformer/USRawData.h:24),
 *    beamformed / envelope images [depth][scanline] (scanline fastest, RxBeamformerCuda.cu:321),
 *    delayed channel data [scanline][channel][depth] (RawDelay.cu:307).
 */
#ifndef SUPRA_B200_H
#define SUPRA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status, dtypes, streams */

#define SB_OK 0
#define SB_ERR_INVALID_ARG (-1)   /* bad pointer, size, enum or parameter range */
#define SB_ERR_CUDA (-2)          /* a CUDA runtime call failed (message has the CUDA error) */
#define SB_ERR_UNSUPPORTED (-3)   /* dtype / configuration combination not implemented */
#define SB_ERR_NO_MEMORY (-4)     /* device or host allocation failed */
#define SB_ERR_TIMEOUT (-5)       /* a bounded device-side wait gave up (persistent kernels) */
#define SB_ERR_NOT_READY (-6)     /* plan used before it was fully initialised */

typedef enum sb_dtype {
    SB_INT16 = 1,      /* SUPRA TypeInt16 */
    SB_FLOAT32 = 2,    /* SUPRA TypeFloat */
    SB_UINT8 = 3,      /* SUPRA TypeUint8 */
    SB_COMPLEX64 = 4,  /* interleaved (re, im) float pairs; extension, no SUPRA counterpart */
    SB_UINT16 = 5      /* SUPRA TypeUint16 (MV output type list) */
} sb_dtype;

typedef void* sb_stream; /* a cudaStream_t */

const char* sb_last_error(void);
int sb_version(int* major, int* minor);

/* ---------------------------------------------------------------- geometry */

/* Window types, same numbering as SUPRA's WindowType (Beamformer/WindowFunction.h:37-44). */
typedef enum sb_window {
    SB_WINDOW_RECTANGULAR = 0,
    SB_WINDOW_HANN = 1,
    SB_WINDOW_HAMMING = 2,
    SB_WINDOW_GAUSS = 3
} sb_window;

/* Transmit reference of one receive scanline. Byte-compatible with
 * ScanlineRxParameters3D::TransmitParameters (SupraLib/USImageProperties.h:52-57). */
typedef struct sb_tx_params {
    uint16_t first_active_element[2]; /* x, y element index of the first active element */
    uint16_t last_active_element[2];  /* x, y; the reference loops use `<`, so this one is skipped */
    uint16_t tx_scanline_idx;         /* transmit event whose channel data this scanline uses */
    uint16_t _pad[3];
    double initial_delay_s;           /* [s] */
} sb_tx_params;

/* Receive scanline, byte-compatible with ScanlineRxParameters3D (SupraLib/USImageProperties.h:43-95),
 * so a std::vector<ScanlineRxParameters3D> can be passed as-is. Positions in mm; direction in the
 * reference's swapped axis order {lateral x, depth, elevation} (Beamformer/Beamformer.cpp:1062-1063). */
typedef struct sb_scanline_rx {
    double position[3];
    double direction[3];
    double tx_weights[4];
    sb_tx_params tx[4];
    double max_element_distance[2]; /* mm, used to normalise the receive window */
} sb_scanline_rx;

/* Receive geometry: what RxBeamformerParameters + USRawData hand to RxBeamformerCuda
 * (Beamformer/RxBeamformerParameters.h:38-112, Beamformer/USRawData.h:24-80). */
typedef struct sb_geometry {
    uint32_t num_elements;        /* transducer elements */
    uint32_t element_layout[2];   /* x, y; 2D probes have y = 1 */
    uint32_t num_channels;        /* received channels per transmit */
    uint32_t num_samples;         /* samples per channel */
    uint32_t num_tx;              /* transmit events (rows of the raw data) */
    uint32_t num_rx;              /* receive scanlines = rx_layout[0] * rx_layout[1] */
    uint32_t rx_layout[2];        /* x, y; 3D when both > 1 */
    uint32_t num_depths;          /* receive depths per scanline */
    double sampling_frequency_hz; /* dt = 1 / fs */
    const float* element_x_mm;    /* [num_elements] element centre x (RxBeamformerParameters m_rxElementXs) */
    const float* element_y_mm;    /* [num_elements] element centre elevation (m_rxElementYs) */
    const float* depths_mm;       /* [num_depths]   receive depths (m_rxDepths) */
    const sb_scanline_rx* scanlines;      /* [num_rx] */
    const int32_t* element_to_channel;    /* optional [num_elements]; -1 = not connected; NULL = e % num_channels */
} sb_geometry;

/* ---------------------------------------------------------------- window + FIR design (host) */

/* 64-entry (or n-entry) receive window LUT normalised to its maximum (Beamformer/WindowFunction.cpp:18-49). */
int sb_window_lut(int window_type, float window_parameter, uint32_t num_entries, float* out_host);

/* FIR design by the window method; type: 0 low-pass, 1 high-pass, 2 band-pass, 3 Hilbert;
 * window: 0 rectangular, 1 Hann, 2 Hamming, 3 Kaiser (SupraLib/utilities/FirFilterFactory.h:58-230). */
int sb_fir_design(uint32_t length, int type, int window, double sampling_frequency, double frequency,
                  double bandwidth, float* out_host);

/* ---------------------------------------------------------------- delay-and-sum */

typedef struct sb_das_plan sb_das_plan;

/* Replaces RxBeamformerCuda(const RxBeamformerParameters&) (Beamformer/RxBeamformerCuda.cu:24-52):
 * copies the geometry to the device. Host pointers in `geometry` are read during the call only. */
int sb_das_plan_create(const sb_geometry* geometry, sb_das_plan** plan);
int sb_das_plan_destroy(sb_das_plan* plan);

/* Replaces RxBeamformerCuda::performRxBeamforming<ChannelDataType, ImageDataType>
 * (Beamformer/RxBeamformerCuda.cu:540-663) with sampleBeamformer = DelayAndSum.
 * rf: [num_tx][num_channels][num_samples] (SB_INT16 or SB_FLOAT32).
 * out: [num_depths][num_rx] (SB_FLOAT32 or SB_INT16, clamped as clampCast).
 * The speed of sound is an argument: no host round trip of the geometry when it changes
 * (RxBeamformerCuda.cu:58-107 copies every buffer D->H->D). 2D or 3D is chosen from rx_layout. */
int sb_das_run(const sb_das_plan* plan, const void* rf, int rf_dtype, void* out, int out_dtype,
               double f_number, double speed_of_sound_mm_s, int window_type, float window_parameter,
               int interpolate_transmits, int32_t additional_offset, sb_stream stream);

/* Sample beamformers (RxBeamformerCuda::RxSampleBeamformer, Beamformer/RxBeamformerCuda.h:31-36, and the
 * BeamformingNode parameter "beamformerType", Beamformer/BeamformingNode.cpp:46). */
#define SB_BF_DELAY_AND_SUM 0        /* "DelayAndSum" */
#define SB_BF_DELAY_AND_STDDEV 1     /* "DelayAndStdDev" (Beamformer/RxSampleBeamformerDelayAndStdDev.h) */
#define SB_BF_COHERENCE_FACTOR_DAS 2 /* "CoherenceFactorDelayAndSum" (...CoherenceFactorDelayAndSum.h) */
#define SB_BF_TEST_SIGNAL 3          /* "TestSignal" (...TestSignal.h): a geometric phantom, no RF read */

/* RxBeamformerCuda::performRxBeamforming(sampleBeamformer, ...) (Beamformer/RxBeamformerCuda.cu:540-662):
 * sb_das_run with the sample beamformer chosen. SB_BF_DELAY_AND_SUM is sb_das_run itself; the others
 * follow the reference's reducers bit for bit in IEEE float semantics (2D and 3D, highest-weight or
 * interpolated transmits, element-to-channel map). */
int sb_das_run_beamformer(const sb_das_plan* plan, int sample_beamformer, const void* rf, int rf_dtype, void* out,
                          int out_dtype, double f_number, double speed_of_sound_mm_s, int window_type,
                          float window_parameter, int interpolate_transmits, int32_t additional_offset, sb_stream stream);

/* HilbertEnvelope::computeHilbertEnvelope (Beamformer/HilbertEnvelope.cu:127-207): the envelope of the
 * analytic signal along each scanline, |x + i H x| with H the circular discrete Hilbert transform of
 * the whole line (the reference's FFT, positive-frequency doubling and inverse FFT), for any number of
 * samples. The plan holds the transform's kernel for num_samples; images are [num_samples][num_scanlines]
 * (SB_INT16 or SB_FLOAT32 in and out; the reference's decimation parameter is not applied, as there). */
typedef struct sb_analytic_plan sb_analytic_plan;
int sb_analytic_plan_create(uint32_t num_samples, sb_analytic_plan** plan);
int sb_analytic_plan_destroy(sb_analytic_plan* plan);
int sb_analytic_env_run(const sb_analytic_plan* plan, const void* in, int in_dtype, void* out, int out_dtype,
                        uint32_t num_scanlines, sb_stream stream);

/* TemporalFilter::filter (Beamformer/TemporalFilter.cu:48-110): out[i] = clampCast(sum_k w_k x_k[i] / sum_k w_k)
 * over num_images device images of numel elements each (images[0] the oldest, the node's queue order),
 * in float as the reference (weights given in double, converted to float; NULL = all 1, the node's
 * weights). num_images in [1, 50]; in/out dtype SB_INT16 or SB_FLOAT32. images is a host array of
 * device pointers. */
int sb_temporal_filter_run(const void* const* images, uint32_t num_images, const double* weights, int in_dtype,
                           void* out, int out_dtype, uint64_t numel, sb_stream stream);

/* ---- Recorded raw data (SUPRA's mock format) ------------------------------------------------------
 * Metadata: RxBeamformerParameters::readMetaDataForMock / writeMetaDataForMock
 * (Beamformer/RxBeamformerParameters.cpp:93-450), ".mock" (ASCII) or ".json" by suffix, parsed with the
 * reference's number types (float fields as float, the JSON depths derived from depth and rxNumDepths).
 * Frames: UltrasoundInterfaceRawDataMock (SupraLib/InputOutput/UltrasoundInterfaceRawDataMock.cpp:47-204),
 * int16 [num_tx][num_channels][num_samples] frames back to back in each data file. */
typedef struct sb_mock_meta sb_mock_meta;
typedef struct sb_mock_reader sb_mock_reader;

int sb_mock_meta_read(const char* filename, sb_mock_meta** meta);
int sb_mock_meta_destroy(sb_mock_meta* meta);
/* The geometry of the metadata (pointers into `meta`, valid until it is destroyed; no channel map). */
int sb_mock_meta_geometry(const sb_mock_meta* meta, sb_geometry* geometry, double* depth_mm,
                          double* speed_of_sound_mm_s);
/* writeMetaDataForMock: the JSON metadata of a geometry (element positions, scanlines, sizes, depth). */
int sb_mock_write_json(const char* filename, const sb_geometry* geometry, double depth_mm, double speed_of_sound_mm_s);
/* A replay of the frame files (comma-separated names, as the node parameter "mockDataFilename"): frames
 * in file order, file after file, wrapping; stream_sequence_once ends after the last frame of the last
 * file; single_image repeats the first frame. A reader thread fills page-locked buffers ahead. */
int sb_mock_reader_create(const sb_mock_meta* meta, const char* data_filenames, int single_image,
                          int stream_sequence_once, sb_mock_reader** reader);
/* Frame bytes, number of files and frames per file (sequence_lengths holds num_sequences entries). */
int sb_mock_reader_info(const sb_mock_reader* reader, uint64_t* frame_bytes, uint32_t* num_sequences,
                        uint64_t* sequence_lengths);
/* Copies the next frame into device_frame (frame_bytes, device memory) on `stream` (asynchronous:
 * one cudaMemcpyAsync from a page-locked buffer). *last_frame = 1 for the final frame of a
 * stream-once replay; later calls fail. */
int sb_mock_reader_next(sb_mock_reader* reader, void* device_frame, sb_stream stream, int* last_frame);
int sb_mock_reader_destroy(sb_mock_reader* reader);

/* Allocation-free delay-and-sum, for callers that cannot allocate device memory: hosts that reserve
 * their whole device budget up front and hand out buffers from their own pool (as SUPRA's container
 * pool does), or real-time frame loops that cannot afford cudaMalloc/cudaFree (cudaFree synchronises
 * the device). No counterpart in the reference. Same arguments and result as sb_das_plan_create +
 * sb_das_run + sb_das_plan_destroy, but nothing is allocated: the geometry (host memory, read by
 * copies enqueued on `stream`; if it is page-locked keep it unchanged until the stream has passed this
 * call) is converted into a fixed scratch area in device memory that the library reserves statically
 * (about 0.4 MB per GPU that loads the library, held until the process exits).
 * Limits: num_elements <= SB_DAS_STATIC_MAX_ELEMENTS, num_depths <= SB_DAS_STATIC_MAX_DEPTHS,
 * num_rx <= SB_DAS_STATIC_MAX_SCANLINES; larger geometries are rejected with SB_ERR_INVALID_ARG.
 * The first call on a device looks up the scratch area's device address (once per device); make that
 * first call before any stream capture. A device reset (cudaDeviceReset) after that first call is not
 * supported: the looked-up address would be stale. All calls share the one scratch area: calls whose
 * work overlaps on the GPU (different streams, or threads) race and must be serialised by the caller.
 * Results are bit-identical to sb_das_run's (2D int16 -> float frames run the same single-frame
 * kernel). A staged copy that never arrives raises a flag kept in the scratch area, reported (and
 * cleared) by sb_check_device_errors like the library's other device errors. */
#define SB_DAS_STATIC_MAX_ELEMENTS 1024
#define SB_DAS_STATIC_MAX_DEPTHS 8192
#define SB_DAS_STATIC_MAX_SCANLINES 1024
int sb_das_run_static(const sb_geometry* geometry, const void* rf, int rf_dtype, void* out, int out_dtype,
                      double f_number, double speed_of_sound_mm_s, int window_type, float window_parameter,
                      int interpolate_transmits, int32_t additional_offset, sb_stream stream);

/* Replaces RawDelay::performDelay (Beamformer/RawDelay.cu:556-650): delayed, apodised and weight-
 * normalised channel samples, out [num_rx][num_channels][num_depths]; slots beyond the active
 * aperture are written as 0. */
int sb_rawdelay_run(const sb_das_plan* plan, const void* rf, int rf_dtype, void* out, int out_dtype,
                    double f_number, double speed_of_sound_mm_s, int window_type, float window_parameter,
                    sb_stream stream);

/* ---------------------------------------------------------------- envelope, log, IQ */

typedef struct sb_hilbert_plan sb_hilbert_plan;

/* Replaces HilbertFirEnvelope(filterLength) (Beamformer/HilbertFirEnvelope.cu:63-82). */
int sb_hilbert_plan_create(uint32_t filter_length, sb_hilbert_plan** plan);
int sb_hilbert_plan_destroy(sb_hilbert_plan* plan);
/* Replaces HilbertFirEnvelope::demodulate (HilbertFirEnvelope.cu:84-104): env = sqrt(x^2 + (h*x)^2).
 * in/out [num_samples][num_scanlines]. Even filter lengths read one tap past the end in the
 * reference; here that tap is 0. */
int sb_hilbert_env_run(const sb_hilbert_plan* plan, const void* in, int in_dtype, void* out, int out_dtype,
                       uint32_t num_scanlines, uint32_t num_samples, sb_stream stream);
/* Extension without a reference counterpart: adjoint of sb_hilbert_env_run for FP32 input.
 * grad_env, in, grad_in: [num_samples][num_scanlines]; grad_in is overwritten. */
int sb_hilbert_env_adjoint(const sb_hilbert_plan* plan, const float* in, const float* grad_env, float* grad_in,
                           uint32_t num_scanlines, uint32_t num_samples, sb_stream stream);

/* Replaces LogCompressor::compress (Beamformer/LogCompressor.cu:44-66). */
int sb_logcompress_run(const void* in, int in_dtype, void* out, int out_dtype, size_t num_values,
                       double dynamic_range_db, double gain, double in_max, sb_stream stream);

typedef struct sb_iq_plan sb_iq_plan;
/* Replaces IQDemodulator(fs, fref, cutoff, lowpassLength, bandpassLength) (Beamformer/IQDemodulator.cu:177-202)
 * plus the frequency-compounding list of IQDemodulatorNode (Beamformer/IQDemodulatorNode.cpp:126-165).
 * reference_frequencies / bandwidths / weights have num_filters entries (<= 8); entry 0 is the
 * unfiltered signal, entries >= 1 use Kaiser band-passes. */
int sb_iq_plan_create(double sampling_frequency, double cutoff_frequency, uint32_t lowpass_filter_length,
                      uint32_t bandpass_filter_length, uint32_t num_filters,
                      const double* reference_frequencies, const double* bandwidths, const double* weights,
                      sb_iq_plan** plan);
int sb_iq_plan_destroy(sb_iq_plan* plan);
/* Replaces IQDemodulator::demodulateMagnitudeFrequencyCompounding (IQDemodulator.cu:215-345):
 * real magnitude output [num_samples / decimation][num_scanlines]. */
int sb_iq_magnitude_run(const sb_iq_plan* plan, const void* in, int in_dtype, void* out, int out_dtype,
                        uint32_t num_scanlines, uint32_t num_samples, uint32_t decimation, sb_stream stream);

/* Extension without a reference counterpart: complex baseband IQ. Mixes with exp(-j 2 pi f n / fs),
 * low-passes with a Hamming-window FIR of lowpass_length taps (cutoff `cutoff_frequency`) and keeps
 * every `decimation`-th sample. out: SB_COMPLEX64 [num_samples / decimation][num_scanlines]. */
int sb_iq_complex_run(const void* in, int in_dtype, void* out, uint32_t num_scanlines, uint32_t num_samples,
                      double sampling_frequency, double mixing_frequency, double cutoff_frequency,
                      uint32_t lowpass_length, uint32_t decimation, sb_stream stream);

/* ---------------------------------------------------------------- scan conversion */

typedef struct sb_scan_plan sb_scan_plan;

/* Replaces ScanConverter::updateInternals (Beamformer/ScanConverter.cu:513-815). scanlines is the
 * layout_x x layout_y grid of the reference's (*scanlines)[x][y], flattened with x fastest
 * (index x + y * layout_x, the order of sb_geometry.scanlines). depth_mm is the image depth,
 * num_samples the samples per scanline. Tables are built on the host (2D, double precision,
 * serial order: on a shared scanline edge the higher quad index wins) or on the device (3D). */
int sb_scan_plan_create(const sb_scanline_rx* scanlines, uint32_t layout_x, uint32_t layout_y,
                        uint32_t num_samples, double depth_mm, double resolution_mm, sb_scan_plan** plan);
int sb_scan_plan_destroy(sb_scan_plan* plan);
int sb_scan_image_size(const sb_scan_plan* plan, uint32_t size_xyz[3]);
/* Host-only 2D table build (no device memory touched): size_xyz receives the image size; when all
 * table pointers are non-NULL they are filled (each size_x * size_y entries). Same tables as
 * sb_scan_plan_create builds for 2D layouts. */
int sb_scan_tables_2d_host(const sb_scanline_rx* scanlines, uint32_t layout_x, uint32_t num_samples, double depth_mm,
                           double resolution_mm, uint32_t size_xyz[3], uint8_t* mask, uint32_t* sample_idx,
                           float* weight_x, float* weight_y);
/* Host copies of the mask / sampleIdx / weightX / weightY / weightZ tables (any pointer may be NULL). */
int sb_scan_copy_tables(const sb_scan_plan* plan, uint8_t* mask, uint32_t* sample_idx, float* weight_x,
                        float* weight_y, float* weight_z);
/* Replaces ScanConverter::convert (ScanConverter.cu:436-495): in [num_samples][scanlines] -> image. */
int sb_scan_run(const sb_scan_plan* plan, const void* in, int in_dtype, void* out, int out_dtype,
                sb_stream stream);

/* HilbertFirEnvelope -> LogCompressor -> ScanConverter (2D or 3D): FP32 RF [num_samples][scanlines]
 * in, image out (SB_UINT8 or SB_FLOAT32). The log-compressed envelope is computed once per input
 * sample into a float image owned by the scan plan (num_samples x scanlines, allocated by
 * sb_scan_plan_create; 1 MB for a 2048 x 128 frame, which stays in L2), then gathered through the
 * tables. Two launches on `stream`; calls on one plan must not overlap. */
int sb_env_log_scan_run(const sb_hilbert_plan* hilbert, const sb_scan_plan* scan, const float* rf,
                        void* out, int out_dtype, double dynamic_range_db, double gain, double in_max,
                        sb_stream stream);

/* ---------------------------------------------------------------- minimum variance */

typedef struct sb_mv_stats {
    uint64_t systems;        /* linear systems solved */
    uint64_t fp64_systems;   /* systems re-solved in FP64 (condition estimate above threshold) */
    float max_condition_estimate;
} sb_mv_stats;

/* Replaces RxBeamformerMV::performRxBeamforming (Beamformer/RxBeamformerMV.cu:382-622).
 * raw_delayed: [num_scanlines][num_channels][num_samples] as written by sb_rawdelay_run
 *   (SB_FLOAT32 real, or SB_COMPLEX64 for the complex extension).
 * out: [num_samples][num_scanlines] (SB_FLOAT32 / SB_INT16 real, SB_COMPLEX64 for complex input).
 * subarray_size 0 means num_channels / 2 (as the reference). loading_scale multiplies the reference's
 * diagonal loading trace(R)/L (1.0 = reference). Systems whose Cholesky condition estimate exceeds
 * fp64_threshold are solved again in FP64 (<= 0 disables). stats_device may be NULL. */
int sb_mv_run(const void* raw_delayed, int in_dtype, void* out, int out_dtype, uint32_t num_scanlines,
              uint32_t num_channels, uint32_t num_samples, uint32_t subarray_size, uint32_t temporal_smoothing,
              double subarray_scaling_power, int compute_means, float loading_scale, float fp64_threshold,
              sb_mv_stats* stats_host, sb_stream stream);

/* Replaces RxBeamformerMVpcg::performRxBeamforming (Beamformer/RxBeamformerMVpcg.cu:622-800): the same
 * covariance, smoothing (over +-temporal_smoothing samples clipped only at the record ends: no
 * 2000-sample blocks), loading and weighting as sb_mv_run, with R a = 1 solved by Jacobi-preconditioned
 * conjugate gradients from a = 1 (residual recomputed every iteration) for max_iterations_override
 * iterations (0: subarray size) or until |r| <= convergence_threshold (BeamformingMVpcgNode passes
 * 10^convergenceThresholdExponent). Real data only (SB_FLOAT32 / SB_INT16 in and out). */
int sb_mv_pcg_run(const void* raw_delayed, int in_dtype, void* out, int out_dtype, uint32_t num_scanlines,
                  uint32_t num_channels, uint32_t num_samples, uint32_t subarray_size, uint32_t temporal_smoothing,
                  uint32_t max_iterations_override, double convergence_threshold, double subarray_scaling_power,
                  int compute_means, float loading_scale, sb_stream stream);

/* ---------------------------------------------------------------- batched, graph-captured DAS + IQ */

typedef struct sb_batch_plan sb_batch_plan;

typedef struct sb_batch_frame {
    const sb_das_plan* probe;  /* geometry of this frame's probe (plans may be shared) */
    const void* rf;            /* device [num_tx][num_channels][num_samples] int16 */
    void* iq_out;              /* device complex64 [num_depths / decimation][num_rx] */
} sb_batch_frame;

typedef struct sb_batch_params {
    double f_number;
    double speed_of_sound_mm_s;
    int window_type;
    float window_parameter;
    double mixing_frequency_hz;
    double cutoff_frequency_hz;
    uint32_t lowpass_length;   /* taps of the decimation low-pass */
    uint32_t decimation;
    int32_t ctas_per_sm;       /* persistent CTAs per SM (0 = default / autotuned) */
    int32_t depth_tile;        /* depths per chunk / per CTA block: 128, 256, 384 or 512 (0 = default) */
    int32_t frames_per_pack;   /* 1: per-frame TMA-staged pipeline; 2, 4 or 8: frames of one probe share the
                                  per-element geometry work (0 = default / autotuned) */
    int32_t staged;            /* with frames_per_pack 2 or 4: 1 stages each depth block's channel samples in
                                  shared memory with cp.async (ctas_per_sm 1 or 2, depth_tile 128); 0: gathers */
} sb_batch_params;

/* Persistent batched DAS + complex IQ over frames of uneven probes in one launch. Frames whose
 * `probe` plans are the same object are grouped: they share delays, apertures and weights. */
int sb_batch_plan_create(const sb_batch_frame* frames, uint32_t num_frames, const sb_batch_params* params,
                         sb_batch_plan** plan);
int sb_batch_plan_destroy(sb_batch_plan* plan);
/* Enqueue one batch. use_graph != 0 replays a captured CUDA graph of the launch sequence. */
int sb_batch_run(sb_batch_plan* plan, int use_graph, sb_stream stream);
/* Optional: write the fused per-frame RF (FP32 [num_depths][num_rx]) too; pass NULL to disable. */
int sb_batch_set_rf_outputs(sb_batch_plan* plan, float* const* rf_out);
/* Time candidate tile shapes on the device and keep the fastest; cache_path (may be NULL) stores
 * the choice per problem signature and is consulted first. Returns the chosen shape. Synchronises. */
int sb_batch_autotune(sb_batch_plan* plan, const char* cache_path, int32_t* ctas_per_sm, int32_t* depth_tile,
                      int32_t* frames_per_pack, int32_t* staged, sb_stream stream);

/* Device-side failure flag shared by the kernels with bounded waits: returns SB_ERR_TIMEOUT if any
 * wait gave up since the last call (and clears the flag when reset != 0). Synchronises the device. */
int sb_check_device_errors(int reset);
/* Self-test of that failure path (no reference counterpart): a kernel waits on an mbarrier that nothing
 * arrives at (arrive = 0) with a limit of `polls` polls, gives up, raises the flag and returns; with
 * arrive = 1 the wait completes. *completed (may be NULL) receives 1 if the wait completed. No fault:
 * the context stays usable. Synchronises `stream`. */
int sb_selftest_bounded_wait(uint32_t polls, int arrive, int* completed, sb_stream stream);
/* Self-test of the Newton square root the 3D delay kernel takes for arguments in [2^-102, FLT_MAX] (bit
 * patterns [0x0C800000, 0x7F800000); no reference counterpart): compares it with the IEEE square root
 * (__fsqrt_rn) on every float whose bit pattern lies in [first_bits, end_bits)
 * (end_bits <= 2^32; equal bits, or NaN for both); *mismatches receives the number of differing results, *first_mismatch (may be
 * NULL) the lowest differing bit pattern (0xFFFFFFFF when none). Synchronises `stream`. */
int sb_selftest_sqrt(uint32_t first_bits, uint64_t end_bits, uint64_t* mismatches, uint32_t* first_mismatch,
                     sb_stream stream);

/* ---------------------------------------------------------------- adjoint DAS */

/* Extension without a reference counterpart. Forward with per-element apodisation:
 *   s = sum_e apod[e] w_e lerp(rf_e, tau_e(c)) / sum_e apod[e] w_e * n_active
 * (apod == NULL means 1, which equals sb_das_run). 2D geometries, highest-weight transmit.
 * rf: FP32 [num_frames][num_tx][num_channels][num_samples]; out: [num_frames][num_depths][num_rx]. */
int sb_das_forward_apod(const sb_das_plan* plan, const float* rf, const float* apod, float* out, uint32_t num_frames,
                        double f_number, double speed_of_sound_mm_s, int window_type, float window_parameter,
                        sb_stream stream);
/* Adjoint of sb_das_forward_apod. Given grad_out [num_frames][num_depths][num_rx] writes grad_rf
 * (same shape as rf; may be NULL), grad_apod [num_elements] (summed over frames; may be NULL) and
 * grad_c (one float: derivative w.r.t. the speed of sound in mm/s, summed over frames; may be NULL).
 * forward_out is the forward result for the same arguments (NULL: recomputed). Outputs are
 * overwritten, not accumulated. The plan keeps the adjoint's device scratch: calls that share a plan
 * must be ordered on one stream. */
int sb_das_adjoint(const sb_das_plan* plan, const float* rf, const float* apod, const float* forward_out,
                   const float* grad_out, float* grad_rf, float* grad_apod, float* grad_c, uint32_t num_frames,
                   double f_number, double speed_of_sound_mm_s, int window_type, float window_parameter,
                   sb_stream stream);

/* ---------------------------------------------------------------- element type conversion */

/* clampCast of n values (SupraLib/utilities/cudaUtility.h:111-147): clamp to the output type's range,
 * then truncate. in: SB_FLOAT32 or SB_INT16; out: SB_FLOAT32, SB_INT16, SB_UINT8 or SB_UINT16. */
int sb_convert_run(const void* in, int in_dtype, void* out, int out_dtype, size_t n, sb_stream stream);

/* ---------------------------------------------------------------- nodes
 * The node layer (C++ API in supra_b200_nodes.hpp) re-hosts SUPRA's receive-path nodes:
 * BeamformingNode, RawDelayNode, BeamformingMVNode, HilbertFirEnvelopeNode, IQDemodulatorNode,
 * LogCompressorNode, ScanConverterNode, with the reference's parameter names, types, ranges and
 * defaults (invalid values fall back to the default and the call returns SB_ERR_INVALID_ARG). These
 * C entry points expose it to non-C++ hosts and tests. */
typedef struct sb_node sb_node;
typedef struct sb_graph sb_graph;
typedef struct sb_record {
    int is_image;      /* 1: USImage [size[2]][size[1]][size[0]], x (scanlines) fastest;
                          0: USRawData [size[2] tx or scanlines][size[1] channels][size[0] samples] */
    int dtype;         /* sb_dtype */
    int state;         /* 0 raw, 1 raw-delayed, 2 RF, 3 envelope, 4 log-compressed, 5 scan-converted */
    uint32_t size[3];
    void* data;        /* device memory, owned by the node / graph until its next call or destruction */
} sb_record;

int sb_node_create(const char* type, const char* node_id, sb_node** node);
int sb_node_destroy(sb_node* node);
int sb_node_set_param(sb_node* node, const char* name, const char* value);
int sb_node_get_param(const sb_node* node, const char* name, char* value, size_t value_len);
int sb_node_param_count(const sb_node* node);
/* name, type (double, uint32_t, int32_t, bool, string, DataType), range ("min..max" or "a|b|c") and
 * default of parameter `index`; each buffer holds `len` bytes. */
int sb_node_param_info(const sb_node* node, int index, char* name, char* type, char* range, char* default_value,
                       size_t len);
int sb_node_type_count(void);
int sb_node_type_name(int index, char* name, size_t len);
/* Runs the node on caller-owned channel data (delayed = 0: [num_tx][num_channels][num_samples] for
 * BeamformingNode / RawDelayNode; delayed = 1: RawDelay output [scanline][channel][depth] for
 * BeamformingMVNode) on `stream`. depth_mm and image_resolution_mm are the image properties the
 * scan converter reads (depth_mm <= 0: the last receive depth). */
int sb_node_process_raw(sb_node* node, const sb_geometry* geometry, const void* data, int dtype, int delayed,
                        uint32_t num_tx, uint32_t num_channels, uint32_t num_samples, double depth_mm,
                        double image_resolution_mm, sb_stream stream, sb_record* out);
/* Runs the node on a caller-owned device image (a USImage [size[2]][size[1]][size[0]], x fastest) in
 * image state `state` (sb_record's codes); geometry (may be NULL) gives the scanline grid the scan
 * converter needs. The data is borrowed: TemporalFilterNode keeps the pointers of its last numImages
 * inputs and reads them again on its next calls, so they must stay valid while they are in its store. */
int sb_node_process_image(sb_node* node, const sb_geometry* geometry, const void* data, int dtype, int state,
                          const uint32_t size[3], double depth_mm, double image_resolution_mm, sb_stream stream,
                          sb_record* out);
/* Runs the node on the last output of `upstream`. */
int sb_node_process_last(sb_node* node, sb_node* upstream, sb_record* out);

/* Graph from the text of a SUPRA XML configuration (inputs, nodes with params, connections). Nodes of
 * types outside the receive path are passed through. */
int sb_graph_create_xml(const char* xml_text, sb_graph** graph);
int sb_graph_destroy(sb_graph* graph);
/* Comma-separated node IDs in processing order; returns their count. */
int sb_graph_chain(const sb_graph* graph, char* ids, size_t len);
int sb_graph_node_get_param(const sb_graph* graph, const char* node_id, const char* name, char* value, size_t len);
int sb_graph_process_raw(sb_graph* graph, const sb_geometry* geometry, const void* data, int dtype, uint32_t num_tx,
                         uint32_t num_channels, uint32_t num_samples, double depth_mm, double image_resolution_mm,
                         sb_stream stream, sb_record* out);
/* For a configuration whose input is UltrasoundInterfaceRawDataMock: the first call opens its
 * mockMetaDataFilename and mockDataFilename (singleImage, streamSequenceOnce as configured); each
 * call copies the next recorded frame to the device and pushes it through the chain. *last_frame = 1
 * on the final frame of a stream-once replay. */
int sb_graph_process_next(sb_graph* graph, double image_resolution_mm, sb_stream stream, int* last_frame,
                          sb_record* out);

#ifdef __cplusplus
}
#endif

#endif /* SUPRA_B200_H */
