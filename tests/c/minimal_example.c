/* Minimal C use of the library: build a 16-ary, 4-level vocabulary from device descriptors, look
 * query descriptors up to leaf word IDs, release the vocabulary.  Compiled (not run) by
 * tests/test_c_header_cpu.py to check that the header is plain C99. */
#include <stdio.h>
#include "rapidbow_b200.h"

int example(const void* dev_desc, uint32_t n_train, uint32_t n_docs, const void* dev_query_desc, uint32_t n_query,
            uint32_t* dev_leaf_ids, void* stream)
{
    rbw_vocabulary* voc = NULL;
    rbw_desc_attr sift = {RBW_DATA_UINT8, RBW_DIST_L2, 128};
    if (rbw_voc_build(sift, 16, dev_desc, n_train, n_docs, 4, NULL, stream, &voc) != RBW_OK) {
        fprintf(stderr, "%s\n", rbw_last_error());
        return 1;
    }
    rbw_voc_lookup(voc, dev_query_desc, n_query, dev_leaf_ids, stream); /* asynchronous on stream */
    rbw_voc_destroy(voc);
    return 0;
}
