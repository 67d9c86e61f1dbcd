// asm_variant_list.h -- every compiled shape of the assembly kernel, one
// line each: RBFB_VARIANT(name, T, GR, GC, NTP, NRHS, P, Q, MIXED, BLOCK, MINB, SMEM, PF)
//   T        compute type of the elimination (double: FP64, float: FP32 + FP64 refinement)
//   GR x GC  lanes per stencil (row groups x column groups), <= 32
//   NTP      padded system size (stencil size + polynomial terms <= NTP)
//   NRHS     right-hand sides compiled in; P, Q degree and PHS exponent
//   MIXED    FP32 factorisation with FP64 refinement
//   BLOCK    threads per CTA; MINB minimum resident CTAs (register budget hint)
//   SMEM     elimination on the matrix in shared memory (large systems) instead
//            of register rows
//   PF       prefetch the next stencil's neighbour data (cp.async) while the
//            current one is solved; off where the extra live state costs the
//            register-bound elimination more than the gather latency it hides
//
// RBFB_BLK_VARIANT(name, T, NMAX, NRHS, P, Q, MIXED, BLOCK, MINB, PB, PF): the
// blocked shared-memory kernel (asm_blocked.cuh), one warp per stencil, any
// system size n <= NMAX, panels of PB columns. RBFB_BLK16_VARIANT: the same
// with half-warp groups, two stencils per warp.
// The build compiles each line as its own translation unit.
RBFB_VARIANT(f64_p4q7_n64_smem, double, 16, 2, 64, 3, 4, 7, false, 32, 1, true, true)
RBFB_VARIANT(f64_p4q7_n80_smem, double, 16, 2, 80, 3, 4, 7, false, 32, 1, true, true)
RBFB_BLK_VARIANT(b64_p3q5_n45_pb8, double, 45, 3, 3, 5, false, 32, 1, 8, true)
RBFB_BLK_VARIANT(b64_p3q5_n45_pb8x3, double, 45, 3, 3, 5, false, 96, 4, 8, true)
RBFB_BLK16_VARIANT(b64_p3q5_n45_pb8_h1, double, 45, 3, 3, 5, false, 32, 1, 8, true)
RBFB_BLK_VARIANT(b64_p3q5_n48_pb8, double, 48, 3, 3, 5, false, 32, 1, 8, true)
RBFB_BLK_VARIANT(b64_p2q3_n32_pb8, double, 32, 3, 2, 3, false, 32, 1, 8, true)
RBFB_BLK_VARIANT(b64_p2q3_n32_pb8x4, double, 32, 3, 2, 3, false, 128, 1, 8, true)
RBFB_BLK_VARIANT(b64_p2q3_n32_r8, double, 32, 8, 2, 3, false, 32, 1, 8, true)
RBFB_BLK_VARIANT(b64_p4q7_n64_pb8, double, 64, 3, 4, 7, false, 32, 1, 8, true)
RBFB_BLK_VARIANT(b64_p4q7_n80_pb8, double, 80, 3, 4, 7, false, 32, 1, 8, true)
RBFB_BLK_VARIANT(bmx_p3q5_n45_pb8, float, 45, 3, 3, 5, true, 32, 1, 8, true)
RBFB_BLK_VARIANT(bmx_p3q5_n45_pb8x3, float, 45, 3, 3, 5, true, 96, 1, 8, true)
RBFB_BLK_VARIANT(bmx_p2q3_n32_pb8, float, 32, 3, 2, 3, true, 32, 1, 8, true)
RBFB_BLK_VARIANT(bmx_p4q7_n80_pb8, float, 80, 3, 4, 7, true, 32, 1, 8, true)
RBFB_VARIANT(f64_p2q3_n32_g16x2, double, 16, 2, 32, 3, 2, 3, false, 64, 6, false, true)
RBFB_VARIANT(f64_p2q3_n32_g16x1, double, 16, 1, 32, 3, 2, 3, false, 64, 1, false, true)
RBFB_VARIANT(f64_p3q5_n48_g16x2, double, 16, 2, 48, 3, 3, 5, false, 64, 1, false, false)
RBFB_VARIANT(mix_p2q3_n32_g16x1, float, 16, 1, 32, 3, 2, 3, true, 64, 1, false, true)
RBFB_VARIANT(mix_p2q3_n32_g16x2, float, 16, 2, 32, 3, 2, 3, true, 64, 1, false, true)
RBFB_VARIANT(mix_p3q5_n48_g16x2, float, 16, 2, 48, 3, 3, 5, true, 64, 4, false, true)
RBFB_VARIANT(mix_p3q5_n48_g16x1, float, 16, 1, 48, 3, 3, 5, true, 64, 1, false, true)
RBFB_VARIANT(mix_p4q7_n64_smem, float, 16, 2, 64, 3, 4, 7, true, 32, 1, true, true)
RBFB_VARIANT(mix_p4q7_n80_smem, float, 16, 2, 80, 3, 4, 7, true, 32, 1, true, true)
