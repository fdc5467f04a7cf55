/* Empty stand-in for AVM v1.0.0's av2/common/quant_common.h, which is not available here.
 * The reference's decision-engine sources include it only for lambda_q8's quantizer table
 * (src/core/quant.cpp:31-39); oracle/ref_shim.cpp defines lambda_q8 from a table the test
 * harness supplies instead. TEST INFRASTRUCTURE ONLY. */
