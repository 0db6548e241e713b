/* bfs.c — CPU oracle: serial breadth-first search (TEST INFRASTRUCTURE ONLY).
 *
 * levels[v] = number of edges on a shortest path from root to v over the CSR graph
 * (rowptr[nv+1], col[E]); unreached vertices keep 0xFFFFFFFF. This is the fixed point the
 * label-correcting async BFS spec converges to, computed the textbook way with a FIFO
 * frontier. Returns the number of reached vertices.
 */
#include <stdint.h>
#include <stdlib.h>

uint32_t oracle_bfs(const uint32_t* rowptr, const uint32_t* col, uint32_t nv, uint32_t root, uint32_t* levels) {
    uint32_t* queue = (uint32_t*)malloc(sizeof(uint32_t) * (nv ? nv : 1));
    uint32_t head = 0, tail = 0;
    for (uint32_t v = 0; v < nv; v++) levels[v] = 0xFFFFFFFFu;
    if (root >= nv) {
        free(queue);
        return 0;
    }
    levels[root] = 0;
    queue[tail++] = root;
    while (head < tail) {
        uint32_t v = queue[head++];
        for (uint32_t e = rowptr[v]; e < rowptr[v + 1]; e++) {
            uint32_t u = col[e];
            if (levels[u] == 0xFFFFFFFFu) {
                levels[u] = levels[v] + 1;
                queue[tail++] = u;
            }
        }
    }
    free(queue);
    return tail;
}
