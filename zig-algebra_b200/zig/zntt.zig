//! Drop-in replacement for the `zig-ntt` module (libs/ntt/src/root.zig) that
//! runs every transform on a B200 through libzntt_cuda.so (include/zntt.h).
//!
//! The seven public functions keep zig-ntt's names, parameters and error
//! names; the error sets gain `DeviceError` and `OutOfMemory` (a GPU can fail
//! where a CPU loop cannot).  `F` must be BN254-Fr or BLS12-381-Fr with
//! zig-field's `BigField` layout (four u64 Montgomery limbs at offset 0), or
//! Goldilocks or BabyBear with its `SmallField` layout (one canonical u64,
//! `value`); any other field is a compile error, since there is deliberately
//! no CPU path.
//!
//! Written for Zig 0.16.0 (the reference's toolchain); it was not compiled
//! in the environment this library was built in, which has no Zig.

const std = @import("std");

const ZStage = extern struct {
    ptr: [*]const u64,
    len: usize,
};

extern fn zntt_init(device: c_int) c_int;
extern fn zntt_bit_reverse(data: [*]u64, len: usize) c_int;
extern fn zntt_bit_reverse_small(data: [*]u64, len: usize) c_int;
extern fn zntt_ntt(field: c_int, data: [*]u64, len: usize, log_n: usize, root: *const [4]u64) c_int;
extern fn zntt_intt(field: c_int, data: [*]u64, len: usize, log_n: usize, root: *const [4]u64) c_int;
extern fn zntt_precompute_twiddles(field: c_int, log_n: usize, root: *const [4]u64, stage_out: [*]const [*]u64) c_int;
extern fn zntt_free_twiddles(field: c_int, stages: [*]const ZStage, num_stages: usize) void;
extern fn zntt_ntt_with_twiddles(field: c_int, data: [*]u64, len: usize, log_n: usize, stages: [*]const ZStage, num_stages: usize) c_int;
extern fn zntt_intt_with_twiddles(field: c_int, data: [*]u64, len: usize, log_n: usize, stages: [*]const ZStage, num_stages: usize) c_int;
extern fn zntt_poly_mul(field: c_int, a: [*]const u64, a_len: usize, b: [*]const u64, b_len: usize, max_degree: usize, out: [*]u64, out_degree: *i64) c_int;

const BN254_FR: u512 = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001;
const BLS12_381_FR: u512 = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001;
const GOLDILOCKS: u64 = 0xFFFFFFFF00000001;
const BABYBEAR: u64 = 0x78000001;

/// `F` is a SmallField (one canonical u64 per element) rather than a BigField.
fn isSmall(comptime F: type) bool {
    return comptime @hasField(F, "value") and @sizeOf(F) == 8;
}

/// The library's field id for `F`, checked at compile time.
fn fieldId(comptime F: type) c_int {
    comptime {
        if (isSmall(F)) {
            if (@offsetOf(F, "value") != 0) @compileError("zig-ntt on B200 needs SmallField's u64 layout");
            if (F.MODULUS == GOLDILOCKS) return 2;
            if (F.MODULUS == BABYBEAR) return 3;
            @compileError("zig-ntt on B200 supports Goldilocks and BabyBear among the small fields");
        }
        if (@sizeOf(F) != 32 or @offsetOf(F, "limbs") != 0 or F.NUM_LIMBS != 4)
            @compileError("zig-ntt on B200 needs a 4x u64 Montgomery field");
        if (F.MODULUS == BN254_FR) return 0;
        if (F.MODULUS == BLS12_381_FR) return 1;
        @compileError("zig-ntt on B200 supports BN254-Fr, BLS12-381-Fr, Goldilocks and BabyBear");
    }
}

const DeviceFailure = error{ DeviceError, OutOfMemory };

/// zntt_init is idempotent and thread-safe (a mutex inside the library): after
/// the first call it only confirms that the library already runs on device 0,
/// so every entry point calls it and the shim needs no once-guard of its own.
fn ensureInit() DeviceFailure!void {
    if (zntt_init(0) != 0) return error.DeviceError;
}

fn limbs(comptime F: type, data: []F) [*]u64 {
    return @ptrCast(data.ptr);
}

/// A root as the C ABI takes it: four limbs, or a small field's value then zeros.
fn rootLimbs(comptime F: type, root: *const F) [4]u64 {
    if (comptime isSmall(F)) return .{ root.value, 0, 0, 0 };
    return root.limbs;
}

/// zig-ntt's `sizeFromLog` (root.zig:33-36).
fn sizeFromLog(log_n: usize) error{LogTooLarge}!usize {
    if (log_n >= @bitSizeOf(usize)) return error.LogTooLarge;
    return @as(usize, 1) << @intCast(log_n);
}

fn mapStatus(status: c_int) anyerror!void {
    return switch (status) {
        0 => {},
        1 => error.LogTooLarge,
        2 => error.LengthMismatch,
        3 => error.InvalidTwiddles,
        4 => error.InvalidLength,
        5 => error.OutOfMemory,
        else => error.DeviceError,
    };
}

pub fn bitReverse(comptime F: type, data: []F) error{ InvalidLength, DeviceError, OutOfMemory }!void {
    _ = fieldId(F);
    const n = data.len;
    if (n == 0 or (n & (n - 1)) != 0) return error.InvalidLength;
    try ensureInit();
    const status = if (comptime isSmall(F)) zntt_bit_reverse_small(limbs(F, data), n) else zntt_bit_reverse(limbs(F, data), n);
    return @errorCast(mapStatus(status));
}

pub fn ntt(comptime F: type, data: []F, log_n: usize, root: F) error{ LogTooLarge, LengthMismatch, InvalidLength, DeviceError, OutOfMemory }!void {
    const id = fieldId(F);
    const n = try sizeFromLog(log_n);
    if (data.len != n) return error.LengthMismatch;
    try ensureInit();
    return @errorCast(mapStatus(zntt_ntt(id, limbs(F, data), data.len, log_n, &rootLimbs(F, &root))));
}

pub fn intt(comptime F: type, data: []F, log_n: usize, root: F) error{ LogTooLarge, LengthMismatch, InvalidLength, DeviceError, OutOfMemory }!void {
    const id = fieldId(F);
    const n = try sizeFromLog(log_n);
    if (data.len != n) return error.LengthMismatch;
    try ensureInit();
    return @errorCast(mapStatus(zntt_intt(id, limbs(F, data), data.len, log_n, &rootLimbs(F, &root))));
}

/// Allocates the table exactly as zig-ntt does (`log_n` stages, stage s of
/// 2^s elements, from `allocator`); the library fills it on the device and
/// keeps a resident copy that nttWithTwiddles/inttWithTwiddles reuse.
pub fn precomputeTwiddles(comptime F: type, log_n: usize, root: F, allocator: std.mem.Allocator) error{ LogTooLarge, OutOfMemory, DeviceError }![]const []const F {
    const id = fieldId(F);
    _ = try sizeFromLog(log_n);
    const twiddles = try allocator.alloc([]F, log_n);
    errdefer allocator.free(twiddles);
    var made: usize = 0;
    errdefer for (twiddles[0..made]) |t| allocator.free(t);
    var ptrs: [64][*]u64 = undefined;
    var s: usize = 0;
    while (s < log_n) : (s += 1) {
        twiddles[s] = try allocator.alloc(F, @as(usize, 1) << @intCast(s));
        made += 1;
        ptrs[s] = @ptrCast(twiddles[s].ptr);
    }
    try ensureInit();
    try @as(error{ LogTooLarge, OutOfMemory, DeviceError }!void, @errorCast(mapStatus(zntt_precompute_twiddles(id, log_n, &rootLimbs(F, &root), &ptrs))));
    return twiddles;
}

pub fn freeTwiddles(comptime F: type, twiddles: []const []const F, allocator: std.mem.Allocator) void {
    const id = fieldId(F);
    if (twiddles.len > 0 and twiddles.len <= 64) {
        var st: [64]ZStage = undefined;
        for (twiddles, 0..) |t, s| st[s] = .{ .ptr = @ptrCast(t.ptr), .len = t.len };
        zntt_free_twiddles(id, &st, twiddles.len);
    }
    for (twiddles) |t| allocator.free(t);
    allocator.free(twiddles);
}

fn withTwiddles(comptime F: type, data: []F, log_n: usize, twiddles: []const []const F, inverse: bool) error{ LogTooLarge, LengthMismatch, InvalidTwiddles, InvalidLength, DeviceError, OutOfMemory }!void {
    const id = fieldId(F);
    const n = try sizeFromLog(log_n);
    if (data.len != n) return error.LengthMismatch;
    if (twiddles.len != log_n) return error.InvalidTwiddles;
    var st: [64]ZStage = undefined;
    for (twiddles, 0..) |t, s| st[s] = .{ .ptr = @ptrCast(t.ptr), .len = t.len };
    try ensureInit();
    const status = if (inverse)
        zntt_intt_with_twiddles(id, limbs(F, data), data.len, log_n, &st, twiddles.len)
    else
        zntt_ntt_with_twiddles(id, limbs(F, data), data.len, log_n, &st, twiddles.len);
    return @errorCast(mapStatus(status));
}

pub fn nttWithTwiddles(comptime F: type, data: []F, log_n: usize, twiddles: []const []const F) error{ LogTooLarge, LengthMismatch, InvalidTwiddles, InvalidLength, DeviceError, OutOfMemory }!void {
    return withTwiddles(F, data, log_n, twiddles, false);
}

pub fn inttWithTwiddles(comptime F: type, data: []F, log_n: usize, twiddles: []const []const F) error{ LogTooLarge, LengthMismatch, InvalidTwiddles, InvalidLength, DeviceError, OutOfMemory }!void {
    return withTwiddles(F, data, log_n, twiddles, true);
}

/// `Polynomial(F, max_degree).mul` (libs/poly/src/poly.zig:197-212) on the GPU, for zig-poly
/// to call in place of its schoolbook loop when the degrees are large.  `P` is the
/// `Polynomial(F, max_degree)` type (fields `coeffs: [MAX_DEGREE + 1]F` and `degree: i32`);
/// the result is the same value, normalized, with the same `DegreeTooLarge` rule.
pub fn polyMul(comptime P: type, a: P, b: P) error{ DegreeTooLarge, DeviceError, OutOfMemory }!P {
    const F = @TypeOf(a.coeffs[0]);
    const id = fieldId(F);
    if (a.degree < 0 or b.degree < 0) return P.zero();
    if (a.degree + b.degree > P.MAX_DEGREE) return error.DegreeTooLarge;
    try ensureInit();
    var r = P.zero();
    var deg: i64 = -1;
    const status = zntt_poly_mul(id, @ptrCast(&a.coeffs), @intCast(a.degree + 1), @ptrCast(&b.coeffs),
        @intCast(b.degree + 1), P.MAX_DEGREE, @ptrCast(&r.coeffs), &deg);
    if (status == 13) return error.DegreeTooLarge;
    try @as(DeviceFailure!void, @errorCast(mapStatus(status)));
    r.degree = @intCast(deg);
    return r;
}
