/*
 * blade_b200 C ABI: the drop-in boundary of the B200-native beamform ->
 * channelize -> detect path.
 *
 * Every entry point takes raw device pointers, shape integers, configuration
 * scalars and a CUDA stream (a cudaStream_t; NULL is the legacy default stream),
 * enqueues its work asynchronously on that stream, and returns a status code
 * that mirrors Blade::Result (reference include/blade/macros.hh:31-48):
 * 0 = SUCCESS, 1 = ERROR (bad shape or configuration, nothing enqueued),
 * 2 = CUDA_ERROR (a launch failed), 3 = ASSERTION_ERROR.  The message of the
 * last failure on the calling thread is returned by blade_last_error().
 *
 * Layouts are the reference's, row-major with the last axis innermost:
 *   ArrayShape  [A, F, T, P]     (include/blade/memory/custom.hh:10-53)
 *   PhasorShape [B, A, F, 1, P]  (include/blade/memory/custom.hh:55-103)
 *   DelayShape  [B, A]           (include/blade/memory/custom.hh:105-138)
 * Complex values are interleaved (re, im) pairs of the scalar type.
 */
#ifndef BLADE_B200_H
#define BLADE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* blade_stream_t; /* same type as cudaStream_t */

#if defined(__GNUC__)
#define BLADE_API __attribute__((visibility("default")))
#else
#define BLADE_API
#endif

/* Status codes (Blade::Result, include/blade/macros.hh:31-48). */
#define BLADE_SUCCESS 0
#define BLADE_ERROR 1
#define BLADE_CUDA_ERROR 2
#define BLADE_ASSERTION_ERROR 3

/* Element types (the reference's I8, I32, F16, F32, F64, CI8, CF16, CF32, CF64;
 * include/blade/memory/types.hh). */
#define BLADE_I8 1
#define BLADE_I32 2
#define BLADE_F16 3
#define BLADE_F32 4
#define BLADE_F64 5
#define BLADE_CI8 6
#define BLADE_CF16 7
#define BLADE_CF32 8
#define BLADE_CF64 9

/* Message of the last failure on this thread ("" if none). */
BLADE_API const char* blade_last_error(void);

/* ABI version: major * 10000 + minor * 100 + patch. */
BLADE_API int blade_version(void);

/* ---------------------------------------------------------------------------
 * Cast: out[i] = static_cast<OT>(in[i]) over the scalar subtype; n_elements
 * counts elements of the input type (a complex element is two scalars).
 * Complex <-> real casts are rejected with BLADE_ERROR.  Bit-exact.
 * Replaces Modules::Cast<IT,OT>::process, src/modules/cast/base.cc:60-66 and
 * the kernel src/modules/cast/cast.cu:5-12.
 * ------------------------------------------------------------------------- */
BLADE_API int blade_cast(int in_type, int out_type, const void* in, void* out,
               uint64_t n_elements, blade_stream_t stream);

/* ---------------------------------------------------------------------------
 * Phasors from delays, in FP64 with FP64 argument reduction:
 *   phasors[b,a,f,0,p] = exp(-i 2 pi tau[b,a] ((f + freq_start_index) * chan_bw_hz))
 *                      * exp(-i 2 pi tau[b,a] (obs_freq_hz - total_bw_hz / 2))
 *                      * calibrations[a,f,0,p]
 * delays: F64 [B,A] (seconds); calibrations: CF64 [A,F,1,P] or NULL (unit);
 * phasors: CF32 [B,A,F,1,P].
 * Replaces the formula half of Modules::Phasor::ATA<CF32>::process,
 * src/modules/phasor/ata.cc:176-208 (host FP64 loops there).
 * ------------------------------------------------------------------------- */
BLADE_API int blade_phasor_from_delays(const double* delays, const void* calibrations,
                             void* phasors, uint64_t B, uint64_t A, uint64_t F,
                             uint64_t P, double obs_freq_hz, double chan_bw_hz,
                             double total_bw_hz, uint64_t freq_start_index,
                             blade_stream_t stream);

/* ---------------------------------------------------------------------------
 * Plain FP32 CUDA-core beamformer (the drop-in):
 *   out[b,f,t,p] = sum_a in[a,f,t,p] * phasors[b,a,f,0,p]   (no conjugate)
 * in: CF32 [A,F,T,P]; phasors: CF32 [B,A,F,1,P]; out: CF32 [B+inc,F,T,P].
 * incoherent != 0 adds beam B = (sum_a |in * phasors[0]|^2 [sqrt], 0).
 * Any A, B, F, T; P in {1, 2}.
 * Replaces Modules::Beamformer::ATA<CF32,CF32> (src/modules/beamformer/ata.cc:7-74,
 * generic.cc:30-33) and its kernel src/modules/beamformer/beamformer.cu:13-79.
 * ------------------------------------------------------------------------- */
BLADE_API int blade_beamform_f32(const void* in, const void* phasors, void* out,
                       uint64_t B, uint64_t A, uint64_t F, uint64_t T, uint64_t P,
                       int incoherent, int incoherent_sqrt, blade_stream_t stream);

/* ---------------------------------------------------------------------------
 * MeerKAT FP32 beamformer:
 *   out[b,f,t,p] = sum_a in[a,f,t,p] * phasors[b*A + a]   (no conjugate)
 * one weight per (beam, antenna), shared by every channel and polarisation: the
 * first B*A values of the phasor buffer, as the reference kernel reads them.
 * in: CF32 [A,F,T,P]; out: CF32 [B+inc,F,T,P]; incoherent != 0 sizes beam B,
 * which the reference allocates but never writes; here it is zero.
 * Replaces Modules::Beamformer::MeerKAT<CF32,CF32> (src/modules/beamformer/
 * meerkat.cc:8-39) and its kernel src/modules/beamformer/beamformer.cu:81-117.
 * ------------------------------------------------------------------------- */
BLADE_API int blade_beamform_meerkat_f32(const void* in, const void* phasors, void* out,
                               uint64_t B, uint64_t A, uint64_t F, uint64_t T,
                               uint64_t P, int incoherent, blade_stream_t stream);

/* ---------------------------------------------------------------------------
 * Channelizer: [A,F,T,P] CF32 -> [A,F*rate,T/rate,P] CF32,
 *   out[a, f*rate + k, s, p] = fftshift(FFT_rate(in[a, f, s*rate:(s+1)*rate, p]))[k]
 * unnormalised, hand-written FP32 Stockham FFT.  rate = 1 copies (or is a no-op
 * when in == out); rate must be even, T % rate == 0, P in {1, 2}, and every
 * prime factor of rate at most 61.  When rate == T the transform may run in
 * place (in == out).  Rates above 4096 need a workspace of
 * blade_channelize_workspace_size() bytes (NULL otherwise).
 * Replaces Modules::Channelizer<CF32,CF32>::process, src/modules/channelizer/
 * base.cc:122-146 (pre_channelizer kernel channelizer.cu:5-19 + cuFFT), and
 * lifts its rate == T restriction (base.cc:30-35).
 * ------------------------------------------------------------------------- */
BLADE_API uint64_t blade_channelize_workspace_size(uint64_t A, uint64_t F, uint64_t T,
                                         uint64_t P, uint64_t rate);
BLADE_API int blade_channelize(const void* in, void* out, void* workspace,
                     uint64_t A, uint64_t F, uint64_t T, uint64_t P, uint64_t rate,
                     blade_stream_t stream);

/* ---------------------------------------------------------------------------
 * Fused spectrometer: Cast -> Channelizer(rate) -> Polarizer -> Detector ->
 * output Cast in two kernels, [A,F,T,2] CI8 or CF32 in, [A,F*rate,T/(rate*I),
 * out_pols] F32 or F16 out; only the input, an FP32 workspace of
 * blade_spectrometer_workspace_size() bytes and the detector products touch HBM.
 * circular != 0 converts (X, Y) to (X + iY, X - iY) before the detector (the
 * Polarizer's XY -> LR), else the detector sees (X, Y).  rate must be 65536
 * (split 256 x 256), T a multiple of it with at most 16 spectra, I dividing the
 * spectra, out_pols 1 or 4 (as blade_detect).  Same results as the module chain
 * blade_cast, blade_channelize, blade_polarize, blade_detect.
 * Replaces Bundles::Generic::ModeH<IT,OT> (include/blade/bundles/generic/
 * mode_h.hh:55-106), whose channelizer runs rate == T only.
 * ------------------------------------------------------------------------- */
BLADE_API uint64_t blade_spectrometer_workspace_size(uint64_t A, uint64_t F, uint64_t T,
                                           uint64_t P, uint64_t rate);
BLADE_API int blade_spectrometer(int in_type, const void* in, int out_type, void* out,
                       void* workspace, uint64_t A, uint64_t F, uint64_t T, uint64_t P,
                       uint64_t rate, uint64_t integration, uint64_t out_pols,
                       int circular, blade_stream_t stream);

/* ---------------------------------------------------------------------------
 * Polarizer: per dual-pol sample (X, Y) -> (X + iY, X - iY); in may equal out.
 * type in {BLADE_CF32, BLADE_CF16}; n_samples = A*F*T (P must be 2).
 * Replaces Modules::Polarizer::process, src/modules/polarizer/base.cc:61-68
 * and src/modules/polarizer/polarizer.cu:5-25.
 * ------------------------------------------------------------------------- */
BLADE_API int blade_polarize(int type, const void* in, void* out, uint64_t n_samples,
                   blade_stream_t stream);

/* ---------------------------------------------------------------------------
 * Detector: [A,F,T,2] CF32 -> [A,F,T/I,out_pols] F32, deterministic sums.
 * out_pols = 4: (|X|^2, |Y|^2, Re X conj Y, Im X conj Y); 1: Stokes-I.
 * Replaces Modules::Detector<CF32,F32>::process, src/modules/detector/base.cc:
 * 82-85 and src/modules/detector/detector.cu:7-51 (atomicAdd there).
 * ------------------------------------------------------------------------- */
BLADE_API int blade_detect(const void* in, void* out, uint64_t A, uint64_t F, uint64_t T,
                 uint64_t P, uint64_t integration, uint64_t out_pols,
                 blade_stream_t stream);

/* ---------------------------------------------------------------------------
 * Gather: copies block `step` of `multiplier` into out along `axis`:
 *   out.shape = in.shape with shape[axis] *= multiplier,
 *   out[..., i + step * shape[axis], ...] = in[..., i, ...].  Bit-exact.
 * Replaces Modules::Gather::process, src/modules/gather/base.cc:70-111
 * (kernel gather.cu:6-18 or Copy2D).
 * ------------------------------------------------------------------------- */
BLADE_API int blade_gather(uint64_t elem_bytes, const void* in, void* out,
                 const uint64_t shape[4], uint64_t axis, uint64_t multiplier,
                 uint64_t step, blade_stream_t stream);

/* ---------------------------------------------------------------------------
 * Permutation: out.shape[i] = in.shape[indexes[i]]; bit-exact element moves.
 * Replaces Modules::Permutation::process, src/modules/permutation/base.cc:70-73
 * and src/modules/permutation/permutation.cu:6-20.
 * ------------------------------------------------------------------------- */
BLADE_API int blade_permute(uint64_t elem_bytes, const void* in, void* out,
                  const uint64_t shape[4], const uint64_t indexes[4],
                  blade_stream_t stream);

/* ---------------------------------------------------------------------------
 * Duplicate: device-to-device copy of `bytes` bytes.  Bit-exact.
 * Replaces Modules::Duplicate::process, src/modules/duplicate/base.cc:34-37.
 * ------------------------------------------------------------------------- */
BLADE_API int blade_duplicate(const void* in, void* out, uint64_t bytes, blade_stream_t stream);

/* ---------------------------------------------------------------------------
 * Fused FP32 CUDA-core chain Cast -> Beamformer -> Channelizer(rate) -> Detector
 * (Stokes-I), in one pass over the voltages:
 *   out[b, f*rate + k, u, 0] = sum_{s in window u} sum_p |Y[b, f*rate+k, s, p]|^2
 * in_type in {BLADE_CI8, BLADE_CF32}; phasors CF32 [B,A,F,1,P]; P = 2;
 * rate in {1, 2, 4}; out F32 [B, F*rate, T/rate/integration, 1].
 * Composes src/modules/cast/cast.cu, beamformer.cu:13-62, channelizer
 * (channelizer.cu + cuFFT) and detector.cu:34-51 of the reference.
 * ------------------------------------------------------------------------- */
BLADE_API int blade_beamform_detect_f32(int in_type, const void* in, const void* phasors,
                              void* out, uint64_t B, uint64_t A, uint64_t F,
                              uint64_t T, uint64_t P, uint64_t rate,
                              uint64_t integration, blade_stream_t stream);

/* ---------------------------------------------------------------------------
 * Tensor-core (tcgen05, sm_100a) chain CI8 -> Beamformer -> Channelizer(rate)
 * -> Detector (Stokes-I).  CI8 voltages enter the MMA exactly as FP16 (rate 2
 * and 4 DFTs are folded into the operand build, still exact); each CF32 phasor
 * is split into an FP16 hi + lo pair whose two products accumulate in FP32 in
 * tensor memory.
 * blade_beamform_tc_plan_size / _prepare turn phasors CF32 [B,A,F,1,P] into the
 * split operand image ("plan", device memory of plan_size bytes; 0 = shape not
 * supported).  blade_beamform_detect_tc runs the chain;
 * out F32 [B, F*rate, T/rate/I, 1].
 * Limits (blade_beamform_detect_tc_supported() returns 1 when met): P = 2,
 * 1 <= A <= 64, any B (64 beams per pass), T % 128 == 0, rate in {1, 2, 4},
 * I a power of two <= 32.  Input and plan 16-byte aligned, output 4-byte
 * aligned; at rate 1 with I = 8 or 16, a 16-byte aligned output lets each full
 * 64-beam pass use the faster epilogue (outputs agree within FP32 rounding).
 * Composes the same reference stages as blade_beamform_detect_f32.
 * ------------------------------------------------------------------------- */
BLADE_API uint64_t blade_beamform_tc_plan_size(uint64_t B, uint64_t A, uint64_t F, uint64_t P);
BLADE_API int blade_beamform_tc_prepare(const void* phasors, void* plan, uint64_t B,
                              uint64_t A, uint64_t F, uint64_t P,
                              blade_stream_t stream);
BLADE_API int blade_beamform_detect_tc_supported(uint64_t B, uint64_t A, uint64_t F,
                                       uint64_t T, uint64_t P, uint64_t rate,
                                       uint64_t integration);
BLADE_API int blade_beamform_detect_tc(const void* in, const void* plan, void* out,
                             uint64_t B, uint64_t A, uint64_t F, uint64_t T,
                             uint64_t P, uint64_t rate, uint64_t integration,
                             blade_stream_t stream);
/* blade_beamform_prepare_detect_tc: blade_beamform_tc_prepare followed by
 * blade_beamform_detect_tc on the same stream, with the chain launched as a
 * programmatic dependent of the split: its set-up and voltage loads overlap the
 * split, and it reads the plan only after the split has finished.  Same
 * arguments, limits and output as the two calls; `in` must be ready before
 * the call is enqueued (stream order), as for blade_beamform_detect_tc. */
BLADE_API int blade_beamform_prepare_detect_tc(const void* phasors, void* plan,
                             const void* in, void* out, uint64_t B, uint64_t A,
                             uint64_t F, uint64_t T, uint64_t P, uint64_t rate,
                             uint64_t integration, blade_stream_t stream);

/* ---------------------------------------------------------------------------
 * ATA ModeB in the reference's own order (pre-beamformer channelizer, per fine
 * channel phasors), as two launches:
 *
 * blade_prechannelize_cf16: Cast<CI8,CF32> -> Channelizer(rate) -> [Polarizer]
 * of include/blade/bundles/ata/mode_b.hh:99-139 on CI8 [A,F,T,2] voltages, out
 * CF16 [A, F*rate, T/rate, 2]: fftshifted rate-point DFT per spectrum
 * (src/modules/channelizer/channelizer.cu:5-19 + cuFFT), then (X + iY, X - iY)
 * when circular != 0 (src/modules/polarizer/polarizer.cu:17-23).  rate in
 * {1, 2, 4}; every output value is an integer of magnitude <= 1024, exact in FP16
 * (the CF32 module chain computes the same values).
 *
 * blade_beamform_detect_tc_cf16: the tensor-core Beamformer::ATA -> Detector
 * (Stokes-I) chain of blade_beamform_detect_tc at rate 1 on CF16 [A,F,T,2]
 * voltages (e.g. the output above, F counting fine channels) with the phasor
 * image of blade_beamform_tc_prepare for [B,A,F,1,2] phasors; out F32
 * [B,F,T/I,1].  Same shape limits as blade_beamform_detect_tc at rate 1.
 * ------------------------------------------------------------------------- */
BLADE_API int blade_prechannelize_cf16(const void* in, void* out, uint64_t A, uint64_t F,
                             uint64_t T, uint64_t P, uint64_t rate, int circular,
                             blade_stream_t stream);
BLADE_API int blade_beamform_detect_tc_cf16(const void* in, const void* plan, void* out,
                                  uint64_t B, uint64_t A, uint64_t F, uint64_t T,
                                  uint64_t P, uint64_t integration, blade_stream_t stream);
/* blade_beamform_prepare_detect_tc_cf16: blade_beamform_tc_prepare followed by
 * blade_beamform_detect_tc_cf16, the chain launched as a programmatic dependent
 * of the split (as blade_beamform_prepare_detect_tc does for CI8).  `in` must be
 * ready before the call is enqueued. */
BLADE_API int blade_beamform_prepare_detect_tc_cf16(const void* phasors, void* plan,
                             const void* in, void* out, uint64_t B, uint64_t A,
                             uint64_t F, uint64_t T, uint64_t P, uint64_t integration,
                             blade_stream_t stream);

/* Incoherent beam of Beamformer::ATA (src/modules/beamformer/beamformer.cu:64-78,
 * square-rooted because the detector follows, mode_b.hh:146-147) through the
 * Stokes-I detector on CF16 [A,F,T,2] voltages: out[f, u] = sum over the window
 * u of I samples, both polarisations and all antennas of |x|^2 |w[0,a,f,0,p]|^2
 * (phasors CF32 [B,A,F,1,2], beam 0 used); out F32 [F, T/I] (beam row B of a
 * ModeB output).  I a power of two <= 32. */
BLADE_API int blade_incoherent_detect_cf16(const void* in, const void* phasors, void* out,
                                 uint64_t A, uint64_t F, uint64_t T, uint64_t P,
                                 uint64_t integration, blade_stream_t stream);

/* ---------------------------------------------------------------------------
 * Device-side status of the pipelined kernels: every wait inside them is
 * bounded, and a wait that expires records a non-zero code here instead of
 * hanging (the kernel then drains its own work and returns).  Synchronous:
 * reads and clears the word.  The reference's equivalent is the sticky-error
 * peek after each launch (include/blade/module.hh:77-80).
 * ------------------------------------------------------------------------- */
BLADE_API int blade_device_status(uint32_t* status);

/* Exercises the expiry path of those bounded waits: one thread waits on a barrier
 * that nothing completes, gives up after budget_cycles SM clock cycles (1 .. 1e10)
 * and records status 0x20, which the next blade_device_status() returns; the
 * kernel itself returns normally, and later launches are unaffected.  No
 * reference counterpart (a health check for callers that monitor the status). */
BLADE_API int blade_wait_selftest(uint64_t budget_cycles, blade_stream_t stream);

/* ---------------------------------------------------------------------------
 * Geometric delays: the astrometric half of Modules::Phasor::ATA::process
 * (src/modules/phasor/ata.cc:9-173; the reference calls ERFA through
 * radiointerferometryc99, neither vendored), restated from published formulas
 * in FP64: IAU 1982 sidereal time, IAU 1976 precession, the leading IAU 1980
 * nutation terms and annual aberration give each source's direction s in the
 * terrestrial frame (polar motion and refraction neglected); then
 *   delays[b, a] = ((r_a - r_ref) . (s_b - s_boresight)) / c   [seconds]
 * (ata.cc:39-47: TPi = (WPi - WPr) / C - (Wi - Wr) / C).
 * antenna_positions: host F64 [A][3] earth-centred (ECEF/ITRF) metres;
 * array_reference_lla: host F64 [3] lon, lat (rad), alt (m) or NULL (it cancels
 * from the differences; only checked); boresight and beam_coordinates (host F64
 * [B][2]): ICRS RA, Dec in radians; julian_date: UTC; dut1: UT1 - UTC seconds;
 * delays: device F64 [B][A], ready for blade_phasor_from_delays.  A + B <= 1024.
 * Parity with ERFA is unpinned (sub-arcsecond model differences).
 * ------------------------------------------------------------------------- */
BLADE_API int blade_geometric_delays(const double* antenna_positions, uint64_t A,
                                     uint64_t reference_antenna, const double* array_reference_lla,
                                     double boresight_ra, double boresight_dec,
                                     const double* beam_coordinates, uint64_t B,
                                     double julian_date, double dut1, double* delays,
                                     blade_stream_t stream);

/* Host only: the unit vector of (ra, dec) in the terrestrial frame at a UTC
 * julian date (the direction blade_geometric_delays projects baselines on). */
BLADE_API int blade_source_direction(double ra, double dec, double julian_date, double dut1,
                                     double direction[3]);

/* ---------------------------------------------------------------------------
 * Launch-shape autotuner.  The reference's only launch knob is a fixed
 * blockSize per module (include/blade/modules/beamformer/generic.hh:20).  Here
 * each tuning call times every launch candidate of one kernel family on the
 * caller's shape (synthetic inputs it allocates and frees itself; CUDA events
 * on `stream`, median of five launches after two warm-ups), checks that each
 * candidate's output is bit-identical to the default candidate's, and stores the
 * fastest identical one in a per-device cache keyed by family and shape.  Every
 * later launch of that shape on that device (through any entry point of the
 * family, eager or captured) uses the stored choice.  Tuning calls synchronise
 * `stream` and allocate; make them at start-up, outside stream capture.
 *
 * Families, their shape keys (shape[0..7]) and launch choices (params[0..3]):
 *   BLADE_TUNE_TC (blade_beamform_detect_tc, blade_beamform_prepare_detect_tc,
 *     blade_beamform_detect_tc_noalloc): key {B, A, F, T, P, rate, integration, 4};
 *     params {mode (0 raw ring of TMA tiles, 1 converter threads load the
 *     voltages, 2 phasor rows in tensor memory), operand stages, raw stages,
 *     tiles per raw stage}.
 *   BLADE_TUNE_F32 (blade_beamform_detect_f32): key {B, A, F, T, P, rate,
 *     integration, in_type}; params {time-group width TG (a CTA covers 4 TG
 *     samples and 1024 / TG beams), 0, 0, 0}.
 *   BLADE_TUNE_SPECTROMETER (blade_spectrometer): key {A, F, T, P, rate,
 *     integration, out_pols, in_type}; params {column-step CTAs per SM, row-step
 *     CTAs per SM, 0, 0}.
 * params[4] = candidates timed, params[5] = candidates whose output differed from
 * the default's (never chosen); params[6..7] = 0.
 * ------------------------------------------------------------------------- */
#define BLADE_TUNE_TC 1
#define BLADE_TUNE_F32 2
#define BLADE_TUNE_SPECTROMETER 3

BLADE_API int blade_beamform_detect_tc_autotune(uint64_t B, uint64_t A, uint64_t F, uint64_t T,
                                                uint64_t P, uint64_t rate, uint64_t integration,
                                                blade_stream_t stream);
BLADE_API int blade_beamform_detect_f32_autotune(int in_type, uint64_t B, uint64_t A, uint64_t F,
                                                 uint64_t T, uint64_t P, uint64_t rate,
                                                 uint64_t integration, blade_stream_t stream);
BLADE_API int blade_spectrometer_autotune(int in_type, int out_type, uint64_t A, uint64_t F,
                                          uint64_t T, uint64_t P, uint64_t rate,
                                          uint64_t integration, uint64_t out_pols,
                                          blade_stream_t stream);

/* What a launch of `shape` in `family` uses now on the current device: params
 * (8 values, as above) and *tuned = 1 with the measured time in *us when it comes
 * from a tuning call, else the default choice with *tuned = 0 and *us = 0. */
BLADE_API int blade_autotune_query(int family, const uint64_t shape[8], uint32_t params[8],
                                   float* us, int* tuned);

/* Forgets every tuned choice (all devices). */
BLADE_API int blade_autotune_clear(void);

/* ---------------------------------------------------------------------------
 * Allocation-free tensor-core chain (no counterpart in the reference).
 * Same computation, arguments and output as blade_beamform_prepare_detect_tc
 * (the split, then the chain overlapping its end), but the phasor image lives in a fixed 8 MiB
 * device array inside this library instead of caller-allocated memory, so the
 * call itself allocates nothing (no cudaMalloc / cudaFree).  It is meant for
 * streaming callers whose device memory is sized once at start-up and whose
 * fixed-cadence loop cannot absorb the device synchronisation of an allocation.
 * Limit: blade_beamform_tc_plan_size(B, A, F, P) <= 8 MiB (e.g. A <= 32,
 * B <= 16 up to 512 channels); larger images are rejected with BLADE_ERROR.
 * The array is part of the library's device code: every process that loads
 * the library holds these 8 MiB on each device it uses, from the module load
 * until exit, whether or not it ever calls this function.
 * The first call on each device (and the first after a cudaDeviceReset) looks
 * up the array's device address (make that first call before any stream
 * capture).  All calls share the one array: calls that overlap on the GPU
 * (different streams, or different host threads) race; serialise them on one
 * stream.  Each call rewrites the whole image it uses.
 * ------------------------------------------------------------------------- */
BLADE_API int blade_beamform_detect_tc_noalloc(const void* in, const void* phasors,
                                               void* out, uint64_t B, uint64_t A,
                                               uint64_t F, uint64_t T, uint64_t P,
                                               uint64_t rate, uint64_t integration,
                                               blade_stream_t stream);

/* ---------------------------------------------------------------------------
 * Adjoint of beamform + Stokes-I detect (no reference counterpart).
 * For L = -sum_{b,f,t,p} |y[b,f,t,p]|^2, y = beamform(in, phasors):
 *   grad[b,a,f,0,p] = dL/d conj(w) = -sum_t y[b,f,t,p] conj(in[a,f,t,p])
 * (beam voltages recomputed tile by tile, never stored).  in CF32 [A,F,T,P],
 * phasors CF32 [B,A,F,1,P], grad CF32 [B,A,F,1,P]; loss (optional, device F64
 * scalar) receives L.  The gradient with respect to (Re w, Im w) is
 * (2 Re grad, 2 Im grad).
 * ------------------------------------------------------------------------- */
BLADE_API int blade_beamform_detect_adjoint(const void* in, const void* phasors, void* grad,
                                  double* loss, uint64_t B, uint64_t A, uint64_t F,
                                  uint64_t T, uint64_t P, blade_stream_t stream);

/* The same gradient and loss on tensor cores: per 128-sample tile the forward
 * y = x w and the contraction over time G += y conj(x) as tcgen05 MMAs with FP16
 * hi/lo splits of voltages, weights and beams and FP32 accumulation in tensor
 * memory; the beams are recomputed per tile and never stored.  Needs P = 2,
 * A <= 32, B <= 32, T % 128 == 0 and 16-byte aligned voltages (else BLADE_ERROR). */
BLADE_API int blade_beamform_detect_adjoint_tc(const void* in, const void* phasors, void* grad,
                                     double* loss, uint64_t B, uint64_t A, uint64_t F,
                                     uint64_t T, uint64_t P, blade_stream_t stream);

/* The same gradient and loss on CUDA cores in FP32, for every shape.
 * blade_beamform_detect_adjoint takes the tensor-core path for 8 <= B and the
 * shapes it supports, this one otherwise (below 8 beams the contraction is
 * GEMV-like and bound by the voltage read, where this kernel is faster). */
BLADE_API int blade_beamform_detect_adjoint_f32(const void* in, const void* phasors, void* grad,
                                      double* loss, uint64_t B, uint64_t A, uint64_t F,
                                      uint64_t T, uint64_t P, blade_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* BLADE_B200_H */
