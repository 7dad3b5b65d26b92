/* gridding oracle: filled in below */
