{
  "targets": [
    {
      "target_name": "s2d_napi",
      "sources": ["s2d_napi.c"],
      "include_dirs": ["../../include"],
      "libraries": ["-L<(module_root_dir)/..", "-ls2d", "-Wl,-rpath,<(module_root_dir)/.."],
      "cflags": ["-std=c11", "-O2", "-Wall"]
    }
  ]
}
