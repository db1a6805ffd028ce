#pragma once
extern "C" {
int mtlg_server_create(mtlg_ctx*, const mtlg_server_opts*, mtlg_server**) { return MTLG_ERR_NOT_SUPPORTED; }
int mtlg_server_destroy(mtlg_server*) { return MTLG_OK; }
int mtlg_server_submit(mtlg_server*, int64_t, int64_t, const int64_t*, const int32_t*, const double*, const double*, int, int, int, int64_t*) { return MTLG_ERR_NOT_SUPPORTED; }
int mtlg_server_step(mtlg_server*) { return MTLG_ERR_NOT_SUPPORTED; }
int mtlg_server_poll(mtlg_server*, int64_t, double*, mtlg_iter_result*) { return MTLG_ERR_NOT_SUPPORTED; }
int mtlg_server_cancel(mtlg_server*, int64_t) { return MTLG_ERR_NOT_SUPPORTED; }
int mtlg_server_stats_get(const mtlg_server*, mtlg_server_stats*) { return MTLG_ERR_NOT_SUPPORTED; }
}
