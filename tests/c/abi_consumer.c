/* A plain C99 consumer of include/tprims_b200.h, compiled and run by
 * tests/test_abi_cpu.py (the counterpart of the reference's C ABI test,
 * crates/tprims-capi/tests/c_abi.rs with tests/c/abi_test.c). It uses only
 * calls that need no GPU: handles, tensor infos, products, the plan report,
 * refusals with their status codes, and N-ary network planning. Exit code 0 on
 * success, else the number of the failed check. */
#include <stdio.h>
#include <string.h>

#include "tprims_b200.h"

#define CHECK(n, cond)                                   \
  do {                                                   \
    if (!(cond)) {                                       \
      fprintf(stderr, "check %d failed: %s\n", n, #cond); \
      return n;                                          \
    }                                                    \
  } while (0)

int main(void) {
  CHECK(1, tprims_abi_version() == 100);
  CHECK(2, TAPP_check_success(TPRIMS_OK) && !TAPP_check_success(TPRIMS_ERR_LABELS));

  TAPP_handle h = 0;
  CHECK(3, TAPP_create_handle(&h) == TPRIMS_OK && h != 0);

  /* D[i,j] = sum_k A[i,k] B[k,j], column-major, i = 4, j = 5, k = 3. */
  const int64_t ea[2] = {4, 3}, sa[2] = {1, 4};
  const int64_t eb[2] = {3, 5}, sb[2] = {1, 3};
  const int64_t ed[2] = {4, 5}, sd[2] = {1, 4};
  TAPP_tensor_info A = 0, B = 0, D = 0;
  CHECK(4, TAPP_create_tensor_info(&A, TAPP_F64, 2, ea, sa) == TPRIMS_OK);
  CHECK(5, TAPP_create_tensor_info(&B, TAPP_F64, 2, eb, sb) == TPRIMS_OK);
  CHECK(6, TAPP_create_tensor_info(&D, TAPP_F64, 2, ed, sd) == TPRIMS_OK);
  CHECK(7, TAPP_get_nmodes(D) == 2);

  const int64_t la[2] = {0, 2}, lb[2] = {2, 1}, ld[2] = {0, 1};
  TAPP_tensor_product p = 0;
  CHECK(8, TAPP_create_tensor_product(&p, h, TAPP_IDENTITY, A, la, TAPP_IDENTITY, B, lb, TAPP_IDENTITY, D, ld,
                                      TAPP_IDENTITY, D, ld, TAPP_DEFAULT_PREC) == TPRIMS_OK);
  char buf[8192];
  const size_t n = tprims_b200_product_report(p, buf, sizeof buf);
  CHECK(9, n > 0 && n < sizeof buf);
  CHECK(10, strstr(buf, "\"m\":4") != NULL && strstr(buf, "\"n\":5") != NULL && strstr(buf, "\"k\":3") != NULL);
  CHECK(11, tprims_b200_product_set_split_k(p, 65) == 1 /* INVALID_ARGUMENT */);
  CHECK(12, tprims_b200_product_set_autotune(p, 1) == TPRIMS_OK);

  /* Refusals: a label of A whose extent disagrees with B's (SHAPE), an
     output-only label (UNSUPPORTED). */
  const int64_t lbad[2] = {0, 1};
  TAPP_tensor_product q = 0;
  CHECK(13, TAPP_create_tensor_product(&q, h, TAPP_IDENTITY, A, lbad, TAPP_IDENTITY, B, lb, TAPP_IDENTITY, D, ld,
                                       TAPP_IDENTITY, D, ld, TAPP_DEFAULT_PREC) != TPRIMS_OK);
  const int64_t e3[3] = {4, 5, 2}, s3[3] = {1, 4, 20}, l3[3] = {0, 1, 7};
  TAPP_tensor_info D3 = 0;
  CHECK(14, TAPP_create_tensor_info(&D3, TAPP_F64, 3, e3, s3) == TPRIMS_OK);
  CHECK(15, TAPP_create_tensor_product(&q, h, TAPP_IDENTITY, A, la, TAPP_IDENTITY, B, lb, TAPP_IDENTITY, D3, l3,
                                       TAPP_IDENTITY, D3, l3, TAPP_DEFAULT_PREC) == TPRIMS_ERR_UNSUPPORTED);
  char msg[256];
  CHECK(16, TAPP_explain_error(TPRIMS_ERR_LABELS, sizeof msg, msg) > 0 && strlen(msg) > 0);
  CHECK(17, strlen(tprims_last_error()) > 0);

  /* A three-tensor network, X[i,j] Y[j,k] Z[k,l] -> W[i,l], greedy path. */
  const int nm[3] = {2, 2, 2};
  const int64_t ex[2] = {4, 3}, ey[2] = {3, 6}, ez[2] = {6, 2}, ew[2] = {4, 2};
  const int64_t lx[2] = {0, 1}, ly[2] = {1, 2}, lz[2] = {2, 3}, lw[2] = {0, 3};
  const int64_t* exts[3] = {ex, ey, ez};
  const int64_t* strs[3] = {NULL, NULL, NULL};
  const int64_t* labs[3] = {lx, ly, lz};
  tprims_b200_network net = 0;
  CHECK(18, tprims_b200_network_create(&net, TAPP_F64, 3, nm, exts, strs, labs, NULL, 2, ew, NULL, lw, 0, NULL) ==
                TPRIMS_OK);
  size_t ws = 0;
  CHECK(19, tprims_b200_network_workspace_size(net, &ws) == TPRIMS_OK && ws > 0);
  CHECK(20, tprims_b200_network_report(net, buf, sizeof buf) > 0 && strstr(buf, "\"greedy_path\":true") != NULL);
  CHECK(21, tprims_b200_network_destroy(net) == TPRIMS_OK);

  CHECK(22, TAPP_destroy_tensor_product(p) == TPRIMS_OK);
  CHECK(23, TAPP_destroy_tensor_info(A) == TPRIMS_OK && TAPP_destroy_tensor_info(B) == TPRIMS_OK &&
                TAPP_destroy_tensor_info(D) == TPRIMS_OK && TAPP_destroy_tensor_info(D3) == TPRIMS_OK);
  CHECK(24, TAPP_destroy_handle(h) == TPRIMS_OK);
  printf("ok\n");
  return 0;
}
