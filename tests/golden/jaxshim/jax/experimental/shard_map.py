def shard_map(*args, **kwargs):
    raise NotImplementedError("shard_map is outside the numpy stand-in")
